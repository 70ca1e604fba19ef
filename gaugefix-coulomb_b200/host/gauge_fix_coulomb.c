/*
 * gauge_fix_coulomb -- drop-in replacement for the reference program of the same
 * name (gauge_fix_coulomb.c:67-211):
 *
 *   gauge_fix_coulomb <config> <gt_out> <ns> <nt> [parameters.par]
 *
 * Same sequence and the same stdout/stderr lines: parameter print-out, "Config
 * from file ... loaded.", the first link before and after reunitarisation, the
 * spatial/temporal plaquettes before and after, the residue at each scheduled
 * check, the sweep count and final residue; the same side file
 * sweeps_to_gaugefix_<ns>x<nt>.txt (appended), the same exit status (0 success,
 * 1 failure), bad parameters falling back to the defaults.  The file formats are
 * those of the reference build's settings.h: FP64 big-endian configuration in,
 * FP64 native-endian gauge transformation out.
 *
 * The work runs on the GPU through libgfc.  Run-time switches (environment; the
 * defaults reproduce the reference):
 *   GFC_PRECISION = exact | fast | mixed   (exact: bit-for-bit the reference update)
 *   GFC_STOP      = reference | every      (check schedule, or test every half-sweep)
 *   GFC_CFG_IN    = f64 | f32              (CONV_CFG_TO_WORKING_PRECISION)
 *   GFC_SWAP_IN   = 1 | 0                  (NEED_BYTE_SWAP_IN)
 *   GFC_GT_OUT    = f64 | f32              (CONV_GT_FROM_WORKING_PRECISION)
 *   GFC_SWAP_OUT  = 0 | 1                  (byte swap of the written G)
 *   GFC_DEVICE    = CUDA device ordinal
 *   GFC_WRITE_CONFIG = 0 | 1               (also write the gauge-fixed configuration to
 *                                           <config>fixed: the writeConfig call the
 *                                           reference's main has commented out,
 *                                           gauge_fix_coulomb.c:185-191; off by default)
 *   GFC_CFG_OUT   = f64 | f32              (CONV_CFG_FROM_WORKING_PRECISION)
 *   GFC_CFG_SWAP_OUT = 0 | 1               (NEED_BYTE_SWAP_OUT)
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "gfc.h"

static const char *env_or(const char *k, const char *d) {
    const char *v = getenv(k);
    return v && *v ? v : d;
}

/* printMatrix3x3 (SU3_ops.c:31-47) */
static void print_matrix(const double *m) {
    printf("{");
    for (int a = 0; a < 3; a++) {
        printf("{");
        for (int b = 0; b < 3; b++) {
            printf("%.*lf + I*(%.*lf)", 18, m[2 * (3 * a + b)], 18, m[2 * (3 * a + b) + 1]);
            if (b != 2) printf(", ");
        }
        if (a != 2) printf("},\n");
    }
    printf("}}\n\n");
}

/* writeSweepsToGaugefix (gauge_fix_coulomb.c:41-65) */
static int write_sweeps(const char *identifier, int ns, int nt, int sweeps) {
    char name[100];
    snprintf(name, sizeof name, "sweeps_to_gaugefix_%dx%d.txt", ns, nt);
    FILE *f = fopen(name, "a+");
    if (!f) {
        fprintf(stderr, "Error opening file %s to record sweeps needed to gaugefix.\n", name);
        return -1;
    }
    fprintf(f, "%s\t%d\n", identifier, sweeps);
    fclose(f);
    return 0;
}

int main(int argc, char *argv[]) {
    const char *config_filename = argc > 1 ? argv[1] : "";
    const char *gt_filename = argc > 2 ? argv[2] : "";
    /* initGeometry takes shorts (geometry.c:184-228) */
    int ns = argc > 3 ? (short)atoi(argv[3]) : 0;
    int nt = argc > 4 ? (short)atoi(argv[4]) : 0;
    int geom_ok = ns > 0 && nt > 0;

    gfc_params p;
    gfc_params_parse_file(argc == 6 ? argv[5] : " ", &p);
    if ((argc != 6 && argc != 5) || !gfc_params_valid(&p) || !geom_ok) {
        fprintf(stderr, "Bad input.\n"
                        "Usage: Input config filename, gt filename, n_SPC, n_T, "
                        "tolerance and omega_OR in this order.\n"
                        "Check that:\n"
                        "1 < omega_OR < 2\n"
                        "n_SPC > 0 and n_T >0\n"
                        "tolerance > 0 \n");
        fprintf(stderr, "\n Provided parameters: \n"
                        "n_SPC: %d \nn_T: %d \n"
                        "omega_OR : %lf \n"
                        "tolerance : %3.2E \n",
                ns, nt, (double)p.omega_OR, p.tolerance);
        fprintf(stderr, "Initializing gauge-fixing parameters to default instead.\n");
        gfc_params_default(&p);
    }
    printf("\nGauge-fixing parameters provided:\n");
    gfc_params_print(&p);

    gfc_options opt;
    gfc_options_default(&opt);
    opt.verbose = 1;
    const char *prec = env_or("GFC_PRECISION", "exact");
    opt.precision = !strcmp(prec, "mixed") ? GFC_PREC_MIXED : !strcmp(prec, "fast") ? GFC_PREC_FP64_FAST
                                                                                    : GFC_PREC_FP64_EXACT;
    opt.stop_rule = !strcmp(env_or("GFC_STOP", "reference"), "every") ? GFC_STOP_EVERY : GFC_STOP_REFERENCE;
    const int in_bytes = !strcmp(env_or("GFC_CFG_IN", "f64"), "f32") ? 4 : 8;
    const int swap_in = atoi(env_or("GFC_SWAP_IN", "1"));
    const int gt_bytes = !strcmp(env_or("GFC_GT_OUT", "f64"), "f32") ? 4 : 8;
    const int swap_out = atoi(env_or("GFC_SWAP_OUT", "0"));
    const int device = atoi(env_or("GFC_DEVICE", "0"));
    const int write_cfg = atoi(env_or("GFC_WRITE_CONFIG", "0"));
    const int cfg_out_bytes = !strcmp(env_or("GFC_CFG_OUT", "f64"), "f32") ? 4 : 8;
    const int cfg_swap_out = atoi(env_or("GFC_CFG_SWAP_OUT", "0"));

    if (!geom_ok) {
        fprintf(stderr, "Loading of file %s failed.\n", config_filename);
        return EXIT_FAILURE;
    }
    const size_t V = (size_t)ns * ns * ns * nt;
    const size_t cfg_bytes = V * 4 * 18 * (size_t)in_bytes;
    /* page-locked when possible (direct DMA); the library stages other memory */
    int pinned = 1;
    void *buf = gfc_host_alloc(cfg_bytes);
    if (buf == NULL) {
        pinned = 0;
        buf = malloc(cfg_bytes);
    }
    if (buf == NULL) {
        fprintf(stderr, "Could not allocate memory for config in file %s.\n", config_filename);
        return EXIT_FAILURE;
    }
#define FREE_BUF() (pinned ? gfc_host_free(buf) : free(buf))
    if (gfc_read_exact(config_filename, buf, cfg_bytes, GFC_FILE_CONFIG)) {
        fprintf(stderr, "Loading of file %s failed.\n", config_filename);
        FREE_BUF();
        return EXIT_FAILURE;
    }
    gfc_ctx *ctx = NULL;
    int rc = gfc_ctx_create(ns, nt, device, opt.precision == GFC_PREC_MIXED ? GFC_CTX_MIXED : 0, &ctx);
    if (rc == GFC_OK) rc = gfc_ctx_upload_links(ctx, buf, in_bytes, swap_in);
    if (rc != GFC_OK) {
        fprintf(stderr, "Could not allocate memory for config in file %s.\n%s\n", config_filename,
                gfc_last_error());
        FREE_BUF();
        if (ctx) gfc_ctx_destroy(ctx);
        return EXIT_FAILURE;
    }
    printf("Config from file %s loaded.\n", config_filename);
    double first[18];
    gfc_ctx_get_link(ctx, 0, 0, first);
    print_matrix(first);

    /* reunitarise right away (gauge_fix_coulomb.c:123-131) */
    unsigned status = 0;
    if (gfc_ctx_reunitarize(ctx) != GFC_OK || gfc_ctx_status(ctx, &status) != GFC_OK || (status & 1u)) {
        fprintf(stderr, "Configuration in file %s could not be reunitarized.\n", config_filename);
        gfc_ctx_destroy(ctx);
        FREE_BUF();
        return EXIT_FAILURE;
    }
    gfc_ctx_get_link(ctx, 0, 0, first);
    print_matrix(first);

    double ps, pt;
    gfc_ctx_plaquette(ctx, &ps, &pt);
    printf("Average trace of spatial plaquettes before gauge transformation: %.10lf\n", ps);
    printf("Average trace of temporal plaquettes before gauge transformation: %.10lf\n", pt);

    gfc_report rep;
    int sweeps = gfc_ctx_fix(ctx, &p, &opt, &rep);
    if (sweeps < GFC_FIX_BAD_PARAMS) {
        fprintf(stderr, "GPU error: %s\n", gfc_last_error());
        gfc_ctx_destroy(ctx);
        FREE_BUF();
        return EXIT_FAILURE;
    }
    gfc_ctx_plaquette(ctx, &ps, &pt);
    printf("Average trace of spatial plaquettes after gauge transformation: %.10lf\n", ps);
    printf("Average trace of temporal plaquettes after gauge transformation: %.10lf\n", pt);

    if (sweeps < 0) {
        gfc_ctx_destroy(ctx);
        FREE_BUF();
        switch (sweeps) {
            case GFC_FIX_NOT_CONVERGED:
                fprintf(stderr, "Configuration in file %s could not be gauge-fixed "
                                "within the maximum number of sweeps passed.\n"
                                "SOR algorithm seems not to work or be slower than "
                                "what the user expected for this particular config. \n",
                        config_filename);
                break;
            case GFC_FIX_BAD_PARAMS:
                fprintf(stderr, "Error in parameters for gauge fixing\n");
                break;
            default:
                break;
        }
        return EXIT_FAILURE;
    }

    printf("Sweeps needed to gauge-fix config from file %s: %d. residue: %3.2E \n", config_filename, sweeps,
           rep.final_residue);
    write_sweeps(config_filename, ns, nt, sweeps);

    /* writeConfig (fields_io.c:405-489) of the gauge-fixed links to <config>fixed, where
       the reference's main has the call commented out (gauge_fix_coulomb.c:185-191) */
    if (write_cfg) {
        const size_t out_size = V * 4 * 18 * (size_t)cfg_out_bytes;
        char *fixed_name = malloc(strlen(config_filename) + 6);
        void *out = out_size <= cfg_bytes ? buf : malloc(out_size);
        int crc = fixed_name && out ? GFC_OK : GFC_ERR_ARG;
        if (crc == GFC_OK) {
            strcpy(fixed_name, config_filename);
            strcat(fixed_name, "fixed");
            crc = gfc_ctx_download_links(ctx, out, cfg_out_bytes, cfg_swap_out);
        }
        if (crc == GFC_OK) crc = gfc_write_all(fixed_name, out, out_size);
        if (crc)
            fprintf(stderr, "Fixed config writing failed for config %s.\n", config_filename);
        else
            printf("U fixed written for config %s.\n", config_filename);
        if (out && out != buf) free(out);
        free(fixed_name);
    }

    /* writeGaugeTransf (fields_io.c:493-565) */
    const size_t gt_size = V * 18 * (size_t)gt_bytes;
    int wrc = gfc_ctx_download_gt(ctx, buf, gt_bytes, swap_out);
    if (wrc == GFC_OK) wrc = gfc_write_all(gt_filename, buf, gt_size);
    if (wrc) {
        fprintf(stderr, "Gauge transformation writing to file %s"
                        "failed for configuration %s .\n",
                gt_filename, config_filename);
    } else {
        printf("G for config %s written to file %s.\n", config_filename, gt_filename);
    }
    gfc_ctx_destroy(ctx);
    FREE_BUF();
    return EXIT_SUCCESS;
}
