/*
 * SCIDAC-binary file access on the host.  The files are headerless arrays of 3x3
 * complex matrices (README.md "Configuration"; fields_io.c:216-565):
 *   configuration: 4V matrices, [t][z][y][x][mu][row][col][re,im]
 *   gauge transf.: V matrices,  [t][z][y][x][row][col][re,im]
 * in FP64 or FP32.  Byte swapping and precision conversion run on the GPU
 * (gfc_ctx_upload_links / gfc_ctx_download_gt); this file only moves bytes and
 * reproduces the reference's size checks and return codes:
 *   loadConfig (fields_io.c:216-305): -1 cannot open, -2 short read,
 *                                     -3 file longer than the lattice
 *   writeGaugeTransf / writeConfig (fields_io.c:405-565): -1 cannot create,
 *                                     -2 short write
 */
#include <stdio.h>
#include <stdlib.h>

#include "gfc.h"

int gfc_read_exact(const char *path, void *buf, size_t bytes, int kind) {
    FILE *f = fopen(path, "rb");
    if (f == NULL) {
        if (kind == GFC_FILE_GT)
            fprintf(stderr, "Error: Problem opening file %s to load gauge transformation.\n", path);
        else
            fprintf(stderr, "Error: Problem opening config file %s.\n", path);
        return -1;
    }
    if (fread(buf, 1, bytes, f) != bytes) {
        if (kind == GFC_FILE_GT)
            fprintf(stderr, "Error: Problem reading file %s to load gauge transformation.\n", path);
        else
            fprintf(stderr, "Error: Reading from file %s.\n", path);
        fclose(f);
        return -2;
    }
    fgetc(f);
    if (!feof(f)) {
        if (kind == GFC_FILE_GT)
            fprintf(stderr, "Error: File has not been read till the end.\nCheck lattice sizes.\n");
        else
            fprintf(stderr, "Error: File has not been read till the end.\n Check lattice sizes.\n");
        fclose(f);
        return kind == GFC_FILE_GT ? -2 : -3;
    }
    fclose(f);
    return 0;
}

int gfc_write_all(const char *path, const void *buf, size_t bytes) {
    FILE *f = fopen(path, "wb");
    if (f == NULL) return -1;
    size_t w = fwrite(buf, 1, bytes, f);
    fclose(f);
    return w == bytes ? 0 : -2;
}

/* byte reversal of 4- or 8-byte words in place (byteSwap, fields_io.c:42-96) */
int gfc_byteswap(void *buf, size_t word_bytes, size_t total_bytes) {
    unsigned char *p = (unsigned char *)buf;
    if (word_bytes == 1) return 0;
    if (word_bytes != 4 && word_bytes != 8) return -1;
    for (size_t o = 0; o + word_bytes <= total_bytes; o += word_bytes)
        for (size_t a = 0, b = word_bytes - 1; a < b; a++, b--) {
            unsigned char t = p[o + a];
            p[o + a] = p[o + b];
            p[o + b] = t;
        }
    return 0;
}
