/*
 * ORACLE -- test infrastructure only.
 *
 * Driver around the reference's own over-relaxation code, compiled from the
 * reference sources where they lie (oracle/Makefile includes src/gauge_fixing.c
 * into this translation unit so that its static gaugefixOverrelaxationLocal,
 * BLACKRED_SWEEP and whenNextConvergenceCheckQ are reachable).  Nothing of the
 * reference is copied here; this file only calls it.
 *
 * Modes:
 *   trace <cfg> <ns> <nt> <params|-> <out_prefix> [max_trace] [trace_every] [dump_sweep]
 *       loadConfig + reunitarizeField + the gaugefixOverrelaxation loop
 *       (gauge_fixing.c:749-826) re-driven half-sweep by half-sweep, recording
 *       calculate_e2 and calculateF after every half-sweep up to max_trace and
 *       after every trace_every-th half-sweep beyond it (large lattices: the
 *       reference's e2 and F are serial loops).  Writes <out_prefix>.trace (text:
 *       sweep e2 F), <out_prefix>.gt (final G, native doubles), <out_prefix>.u
 *       (final U), <out_prefix>.summary and, when the loop passes dump_sweep,
 *       <out_prefix>.gt_dump (G right after that half-sweep and the reunitarisation
 *       that follows it, if one is due).
 *   bench <cfg> <ns> <nt> <half_sweeps> [threads]
 *       times <half_sweeps> half-sweeps of the reference loop body (OpenMP over t,
 *       as gauge_fixing.c:773-787) with omp_get_wtime and prints one line:
 *       "site_updates <n> seconds <s> threads <k>".
 */
#include <omp.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include GAUGE_FIXING_SRC

#include <fields_io.h>
#include <measurement.h>

static int write_doubles(const char *path, const void *p, size_t n) {
    FILE *f = fopen(path, "wb");
    if (!f) return -1;
    size_t w = fwrite(p, sizeof(double), n, f);
    fclose(f);
    return w == n ? 0 : -1;
}

static double wall(void) { return omp_get_wtime(); }

int main(int argc, char **argv) {
    if (argc < 6) {
        fprintf(stderr, "usage: trace|bench ...\n");
        return 2;
    }
    const char *mode = argv[1];
    char *cfg = argv[2];
    initGeometry(atoi(argv[3]), atoi(argv[4]));
    const unsigned V = lattice_param.volume;

    Mtrx3x3 *U = allocate3x3Field(DIM * V);
    Mtrx3x3 *G = allocate3x3Field(V);
    if (!U || !G) return 3;
    if (loadConfig(U, cfg)) return 4;
    reunitarizeField(U, DIM * V);

    if (!strcmp(mode, "bench")) {
        /* bench <cfg> <ns> <nt> <half_sweeps_per_step> [threads] [steps] [warmup] */
        int hs = atoi(argv[5]);
        int threads = argc > 6 && atoi(argv[6]) > 0 ? atoi(argv[6]) : omp_get_num_procs();
        int steps = argc > 7 ? atoi(argv[7]) : 1;
        int warm = argc > 8 ? atoi(argv[8]) : 0;
        ORGaugeFixingParameters p = initParametersORDefault();
        setFieldToIdentity(G, V);
        int sweep = 0;
        for (int k = -warm; k < steps; k++) {
            double t0 = wall();
            for (int j = 0; j < hs; j++, sweep++) {
                #pragma omp parallel for num_threads(threads) schedule(dynamic)
                for (PosIndex t = 0; t < lattice_param.n_T; t++) {
                    PosVec position;
                    position.pos[T_INDX] = t;
                    LOOP_SPATIAL(position) {
                        if (BLACKRED_SWEEP(position, sweep))
                            gaugefixOverrelaxationLocal(U, G, position, p);
                    }
                }
            }
            double t1 = wall();
            if (k >= 0)
                printf("step %d site_updates %.0f seconds %.6f threads %d\n", k, (double)hs * V / 2.0, t1 - t0,
                       threads);
        }
        return 0;
    }

    /* trace */
    if (argc < 7) return 2;
    ORGaugeFixingParameters p = strcmp(argv[5], "-") ? initORGaugeFixingParameters(argv[5])
                                                      : initParametersORDefault();
    const char *prefix = argv[6];
    int max_trace = argc > 7 ? atoi(argv[7]) : 100000;
    int trace_every = argc > 8 ? atoi(argv[8]) : 0;
    int dump_sweep = argc > 9 ? atoi(argv[9]) : -1;
    char path[1024];
    snprintf(path, sizeof path, "%s.trace", prefix);
    FILE *tr = fopen(path, "w");
    if (!tr) return 5;

    setFieldToIdentity(G, V);
    const double plaq_s0 = (double)averagePlaquette(U, "spatial");
    const double plaq_t0 = (double)averagePlaquette(U, "temporal");
    int sweep = 0, rc = 0;
    double res = p.generic_gf.gfix_proxy(U);
    fprintf(tr, "%d %.17e %.17e\n", 0, calculate_e2(U), calculateF(U));
    int due = whenNextConvergenceCheckQ(sweep, res, p);
    while (res > p.generic_gf.tolerance) {
        #pragma omp parallel for num_threads(NUM_THREADS) schedule(dynamic)
        for (PosIndex t = 0; t < lattice_param.n_T; t++) {
            PosVec position;
            position.pos[T_INDX] = t;
            LOOP_SPATIAL(position) {
                if (BLACKRED_SWEEP(position, sweep))
                    gaugefixOverrelaxationLocal(U, G, position, p);
            }
        }
        sweep++;
        if (sweep <= max_trace || (trace_every > 0 && sweep % trace_every == 0)) {
            fprintf(tr, "%d %.17e %.17e\n", sweep, calculate_e2(U), calculateF(U));
            fflush(tr);
        }
        if (sweep == due) {
            double last = res;
            res = p.generic_gf.gfix_proxy(U);
            if (fabs(res - last) / last < 10E-16) { rc = -1; break; }
            else if (res <= p.generic_gf.tolerance) break;
            else due = whenNextConvergenceCheckQ(sweep, res, p);
        }
        if (sweep >= p.generic_gf.max_sweeps_to_fix) { rc = -1; break; }
        if (!(sweep % p.generic_gf.sweeps_to_reunitarization)) {
            reunitarizeField(U, DIM * V);
            reunitarizeField(G, V);
        }
        if (sweep == dump_sweep) {
            snprintf(path, sizeof path, "%s.gt_dump", prefix);
            write_doubles(path, G, (size_t)V * 18);
        }
    }
    if (rc == 0) {
        reunitarizeField(U, DIM * V);
        reunitarizeField(G, V);
    }
    fclose(tr);
    snprintf(path, sizeof path, "%s.gt", prefix);
    write_doubles(path, G, (size_t)V * 18);
    snprintf(path, sizeof path, "%s.u", prefix);
    write_doubles(path, U, (size_t)V * 4 * 18);
    snprintf(path, sizeof path, "%s.summary", prefix);
    FILE *s = fopen(path, "w");
    fprintf(s, "sweeps %d\nrc %d\nfinal_residue %.17e\ne2 %.17e\ntheta %.17e\nF %.17e\n"
               "plaq_spatial %.17e\nplaq_temporal %.17e\nplaq_spatial_0 %.17e\nplaq_temporal_0 %.17e\n",
            rc == 0 ? sweep : rc, rc, p.generic_gf.gfix_proxy(U), calculate_e2(U), calculateTheta(U),
            calculateF(U), (double)averagePlaquette(U, "spatial"), (double)averagePlaquette(U, "temporal"),
            plaq_s0, plaq_t0);
    fclose(s);
    return 0;
}
