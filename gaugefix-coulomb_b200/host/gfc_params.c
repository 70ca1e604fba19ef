/*
 * Gauge-fixing parameters: defaults, validation, the key:value file parser and the
 * parameter print-out, with the reference's semantics and messages
 * (src/gauge_fixing.c:45-244).
 *
 *  - every line is read with a 100-byte fgets, all whitespace is removed, and the
 *    line is split at the first ':' (strtok); lines without a value are ignored,
 *    which makes them comments;
 *  - numbers go through atof and are then converted to the member's type
 *    (omega_OR is a float, the counters unsigned);
 *  - unknown keys print "Unrecognized parameter: <key>." on stderr, an unknown
 *    proxy "Unrecognized gfix_proxy: <value>." and leaves the proxy unchanged;
 *  - invalid values set the error flag; the caller decides what to do.
 * Two spellings the reference's README and print labels use are accepted as well:
 * "max_hits" (for "hits") and "estimate_sweeps_to_gfixprogress".
 */
#include <ctype.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "gfc.h"

void gfc_params_default(gfc_params *p) {
    memset(p, 0, sizeof *p);
    p->omega_OR = 1.95f;
    p->hits = 2;
    p->error = 0;
    p->gfix_proxy = GFC_PROXY_E2;
    p->tolerance = 1E-16;
    p->max_sweeps_to_fix = 100000;
    p->estimate_sweeps_to_gf_progress = 1000;
    p->sweeps_to_reunitarization = 250;
}

int gfc_params_valid(const gfc_params *p) {
    return p->omega_OR >= 1 && p->omega_OR < 2 && p->tolerance > 0 && p->error == 0 &&
           p->sweeps_to_reunitarization > 0;
}

void gfc_params_print(const gfc_params *p) {
    printf("\n");
    printf("max_hits: %u\n", p->hits);
    printf("omega_OR: %lf\n", (double)p->omega_OR);
    printf("\n");
    printf("tolerance: %3.2E\n", p->tolerance);
    printf("max_sweeps_to_fix: %u\n", p->max_sweeps_to_fix);
    printf("estimate_sweeps_to_gfixprogress: %u\n", p->estimate_sweeps_to_gf_progress);
    printf("\n");
    printf("sweeps_to_reunitarization: %u\n", p->sweeps_to_reunitarization);
    printf("\n");
}

static void strip_spaces(char *s) {
    int n = 0;
    for (unsigned k = 0; s[k]; k++)
        if (!isspace((unsigned char)s[k])) s[n++] = s[k];
    s[n] = '\0';
}

int gfc_params_parse_file(const char *path, gfc_params *p) {
    gfc_params_default(p);
    if (path == NULL || !strcmp(path, " ")) {
        printf("No parameter-file detected, using default values.\n");
        return GFC_OK;
    }
    FILE *f = fopen(path, "r");
    char buff[100];
    if (f != NULL) {
        while (fgets(buff, 100, f)) {
            strip_spaces(buff);
            char *key = strtok(buff, ":");
            char *value = strtok(NULL, "\n");
            if (!value) continue;
            if (!strcmp(key, "tolerance")) {
                p->tolerance = atof(value);
            } else if (!strcmp(key, "hits") || !strcmp(key, "max_hits")) {
                p->hits = (unsigned)atof(value);
            } else if (!strcmp(key, "omega_OR")) {
                p->omega_OR = (float)atof(value);
            } else if (!strcmp(key, "max_sweeps_to_fix")) {
                p->max_sweeps_to_fix = (unsigned)atof(value);
            } else if (!strcmp(key, "estimate_sweeps_to_gf_progress") ||
                       !strcmp(key, "estimate_sweeps_to_gfixprogress")) {
                p->estimate_sweeps_to_gf_progress = (unsigned)atof(value);
            } else if (!strcmp(key, "sweeps_to_reunitarization")) {
                p->sweeps_to_reunitarization = (unsigned)atof(value);
            } else if (!strcmp(key, "gfix_proxy")) {
                if (!strcmp(value, "e2"))
                    p->gfix_proxy = GFC_PROXY_E2;
                else if (!strcmp(value, "theta"))
                    p->gfix_proxy = GFC_PROXY_THETA;
                else
                    fprintf(stderr, "Unrecognized gfix_proxy: %s.\n", value);
            } else if (strcmp(key, "\n")) {
                fprintf(stderr, "Unrecognized parameter: %s.\n", key);
            }
        }
        fclose(f);
    } else {
        fprintf(stderr,
                "Gauge-fixing parameter file %s could not be opened. "
                "Using default parameters instead.\n",
                path);
        gfc_params_print(p);
    }
    if (!gfc_params_valid(p)) p->error = 1;
    return GFC_OK;
}
