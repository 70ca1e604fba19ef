// gfc_fast.h -- fast sweep kernels and the drivers that use them.
#pragma once
#include "gfc.h"
#include "gfc_ctx.h"

namespace gfc {
// n fast FP64 half-sweeps (indices first..first+n-1) on the context's u/g, run on the
// two-row working copies (packed before, unpacked after)
int halfsweeps_fast64(gfc_ctx *c, int first, int n, double omega, unsigned hits);
// odd ns, fast arithmetic on two stored rows in the lexicographic layout
int halfsweeps_odd_fast(gfc_ctx *c, int first, int n, double omega, unsigned hits);
int fix_every_sweep_odd_fast(gfc_ctx *c, const gfc_params *p, const gfc_options *o, gfc_report *r);
// GFC_STOP_EVERY driver (FP64 fast or exact update, proxy tested every half-sweep)
int fix_every_sweep(gfc_ctx *c, const gfc_params *p, const gfc_options *o, gfc_report *r);
// FP32 two-row bulk until e2 < switch_e2, then FP64 refinement
int fix_mixed(gfc_ctx *c, const gfc_params *p, const gfc_options *o, gfc_report *r);
}  // namespace gfc
