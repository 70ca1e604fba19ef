// gfc_internal.h -- declarations shared by the library's translation units.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>

#include "gfc_device.cuh"

// bits of the device status word
#define GFC_STATUS_PROJECT_FAIL 1u   // a projectSU3 met a null row (the reference's -1)
#define GFC_STATUS_NAN          2u   // a reduction produced NaN
#define GFC_STATUS_CONVERGED    4u   // a device-side stopping test fired

struct gfc_batch;

namespace gfc {

// Raise a kernel's dynamic shared-memory limit (and prefer shared memory in the
// L1/shared split) on the current device, once per device: a function attribute
// belongs to the device's context.  Host threads racing on one device may both set
// it, which is harmless; the device's bit is set only after the attribute is.
template <typename K>
inline void smem_attr_once(std::atomic<unsigned long long> &done, K kern, size_t bytes) {
    int dev = 0;
    cudaGetDevice(&dev);
    const unsigned long long bit = dev >= 0 && dev < 64 ? 1ull << dev : 0ull;
    if (bit && (done.load(std::memory_order_acquire) & bit)) return;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
    if (bit) done.fetch_or(bit, std::memory_order_release);
}

// ---- exact FP64 kernels (gfc_kernels_exact.cu)
// stop (optional): a device stop word; once set, the launch does nothing
int launch_sweep_exact(double2 *u, double2 *g, const Lat &l, int sweep, double omega, unsigned hits,
                        cudaStream_t s, int shape = 0, const unsigned *stop = nullptr);
int exact_num_shapes();
void launch_reunitarize(double2 *base, uint32_t stride, uint32_t nblk, unsigned *status, cudaStream_t s);
void launch_identity(double2 *g, const Lat &l, cudaStream_t s);
int obs_blocks_per_slice(const Lat &l);
void launch_finalize2(const double *part, const Lat &l, int nbx, double *out, cudaStream_t s, const unsigned *stop);
void launch_obs(const double2 *u, const Lat &l, double *part, double *out, double *slice_out, cudaStream_t s,
                const unsigned *stop = nullptr);
// proxy of out (launch_obs) <= tol sets *stop = sweep (once)
void launch_exact_check(const double *out, const Lat &l, int theta, double tol, int sweep, unsigned *stop,
                        cudaStream_t s);
void launch_functional(const double2 *u, const Lat &l, double *part, double *out, cudaStream_t s);

// ---- layout transforms (gfc_kernels_io.cu)
// Raw file bytes (reference AoS order, elem_bytes 8 or 4, optionally big endian)
// for timeslices [t0, t0+nts) -> SoA FP64 spatial links u and temporal links ut.
// (reunit != 0: each matrix projected to SU(3) as it is stored; failures set status)
void launch_load_links(const void *raw, int elem_bytes, int swap, const Lat &l, uint32_t t0, uint32_t nts,
                       double2 *u, double2 *ut, cudaStream_t s, int reunit = 0, unsigned *status = nullptr);
// SoA FP64 G of timeslices [t0, t0+nts) -> AoS (elem_bytes 8 or 4, optional swap)
void launch_store_gt(const double2 *g, const Lat &l, uint32_t t0, uint32_t nts, int elem_bytes, int swap,
                     void *raw, cudaStream_t s);
// AoS raw G -> SoA FP64 (warm start)
void launch_load_gt(const void *raw, int elem_bytes, int swap, const Lat &l, uint32_t t0, uint32_t nts,
                    double2 *g, cudaStream_t s);
// SoA links (spatial u, temporal ut) of timeslices [t0, t0+nts) -> AoS raw
void launch_store_links(const double2 *u, const double2 *ut, const Lat &l, uint32_t t0, uint32_t nts,
                        int elem_bytes, int swap, void *raw, cudaStream_t s);
// ut(x) <- G(x) ut(x) G(x+t)^dagger  (deferred temporal transform)
void launch_temporal_transform(double2 *ut, const double2 *g, const Lat &l, cudaStream_t s);
// u_d(x) <- G(x) u0_d(x) G(x+d)^dagger for the spatial links (rebuild from originals)
void launch_apply_gt_spatial(double2 *u, const double2 *u0, const double2 *g, const Lat &l, cudaStream_t s);
// applyGaugeTransformationU in the reference's arithmetic, in place (temporal: also ut)
void launch_apply_gt(double2 *u, double2 *ut, const double2 *g, const Lat &l, int temporal, cudaStream_t s);
// format conversions over nblk SoA blocks of `stride` matrices (gfc_fast.cu)
void launch_to_f32(const double2 *src, float4 *dst, uint32_t stride, uint32_t nblk, cudaStream_t s);
void launch_identity32(float4 *g, uint32_t stride, uint32_t nblk, cudaStream_t s);
void launch_pack2(const double2 *src, double2 *dst, uint32_t stride, uint32_t nblk, cudaStream_t s);
void launch_unpack2(const double2 *src, double2 *dst, uint32_t stride, uint32_t nblk, cudaStream_t s);
// seeded synthetic links built on the device (gfc_synth_dev.cu); gtmp is a
// G-sized scratch field (overwritten)
void launch_synth(const Lat &l, uint64_t seed, double scale, double2 *gtmp, double2 *u, double2 *ut,
                  cudaStream_t s);
// plaquette partials: [nt][nbx][2] = (spatial sum, temporal sum) of Re Tr/3
void launch_plaquette(const double2 *u, const double2 *ut, const Lat &l, double *part, double *out,
                      cudaStream_t s);

// ---- batch internals shared with the request server (gfc_batch.cu)
// G of a finalised slot to host memory, staged and copied on stream st; synchronous
int batch_download_gt_on(::gfc_batch *b, int slot, void *host, int elem_bytes, int byteswap, cudaStream_t st);
// map `bytes` of device memory into the batch's slot pool ahead of time
int batch_warm_pool(::gfc_batch *b, size_t bytes);

}  // namespace gfc
