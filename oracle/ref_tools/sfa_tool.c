/* sfa_tool.c -- test-infrastructure helper that moves raw FP64 column blocks
 * in and out of SFA archives through the reference's own single-header SFA
 * library (sfa/format/sfa.h), so the reference CPU stepper can be fed the
 * seeded inputs of the parity tests and its output frames can be read back.
 *
 * Built only by oracle/Makefile into oracle/_ref/ (never shipped, never linked
 * into the product).  Usage:
 *
 *   sfa_tool write OUT.sfa N L dt NCOLS RAW.f64
 *       RAW.f64 holds NCOLS*N^3 little-endian doubles, columns in the
 *       stepper's registration order (12 real, 24 complex or 30 gauged columns,
 *       sfa/sim/scp_sim.c:2862-2897).  Writes one F64 frame at t=0, raw codec.
 *
 *   sfa_tool read IN.sfa FRAME OUT.f64
 *       Decodes frame FRAME (negative counts from the end), converts every
 *       column to FP64 and writes them back to back.  Prints one line per
 *       column: "name semantic component dtype".
 */
#define SFA_IMPLEMENTATION
#include "sfa.h"

#include <stdlib.h>
#include <string.h>

typedef struct { const char *name; int sem, comp; } ColDef;

/* Column names, semantics and components of the complex/gauged stepper's
 * snapshot schema, in registration order (sfa/sim/scp_sim.c:2862-2897). */
static const ColDef kCols[30] = {
    {"phi_x", SFA_POSITION, 0},     {"phi_y", SFA_POSITION, 1},     {"phi_z", SFA_POSITION, 2},
    {"theta_x", SFA_ANGLE, 0},      {"theta_y", SFA_ANGLE, 1},      {"theta_z", SFA_ANGLE, 2},
    {"phi_vx", SFA_VELOCITY, 0},    {"phi_vy", SFA_VELOCITY, 1},    {"phi_vz", SFA_VELOCITY, 2},
    {"theta_vx", SFA_VELOCITY, 3},  {"theta_vy", SFA_VELOCITY, 4},  {"theta_vz", SFA_VELOCITY, 5},
    {"phiim_x", SFA_POSITION, 3},   {"phiim_y", SFA_POSITION, 4},   {"phiim_z", SFA_POSITION, 5},
    {"thetaim_x", SFA_ANGLE, 3},    {"thetaim_y", SFA_ANGLE, 4},    {"thetaim_z", SFA_ANGLE, 5},
    {"phiim_vx", SFA_VELOCITY, 6},  {"phiim_vy", SFA_VELOCITY, 7},  {"phiim_vz", SFA_VELOCITY, 8},
    {"thetaim_vx", SFA_VELOCITY, 9},{"thetaim_vy", SFA_VELOCITY, 10},{"thetaim_vz", SFA_VELOCITY, 11},
    {"th_x", SFA_ANGLE, 6},         {"th_y", SFA_ANGLE, 7},         {"th_z", SFA_ANGLE, 8},
    {"E_x", SFA_VELOCITY, 12},      {"E_y", SFA_VELOCITY, 13},      {"E_z", SFA_VELOCITY, 14},
};

static int do_write(int argc, char **argv) {
    if (argc != 8) { fprintf(stderr, "usage: sfa_tool write OUT N L dt NCOLS RAW\n"); return 2; }
    const char *out = argv[2];
    int N = atoi(argv[3]);
    double L = atof(argv[4]), dt = atof(argv[5]);
    int ncols = atoi(argv[6]);
    if (N < 2 || (ncols != 12 && ncols != 24 && ncols != 30)) { fprintf(stderr, "bad N/NCOLS\n"); return 2; }
    size_t n3 = (size_t)N * N * N;
    double *raw = malloc(sizeof(double) * n3 * ncols);
    FILE *fp = fopen(argv[7], "rb");
    if (!raw || !fp || fread(raw, sizeof(double), n3 * ncols, fp) != n3 * ncols) {
        fprintf(stderr, "cannot read %s\n", argv[7]);
        return 1;
    }
    fclose(fp);
    SFA *s = sfa_create(out, N, N, N, L, L, L, dt);
    if (!s) { fprintf(stderr, "cannot create %s\n", out); return 1; }
    s->flags = SFA_CODEC_RAW;
    for (int c = 0; c < ncols; c++)
        sfa_add_column(s, kCols[c].name, SFA_F64, (uint8_t)kCols[c].sem, (uint8_t)kCols[c].comp);
    sfa_finalize_header(s);
    void *cols[30];
    for (int c = 0; c < ncols; c++) cols[c] = raw + (size_t)c * n3;
    sfa_write_frame(s, 0.0, cols);
    sfa_close(s);
    free(raw);
    return 0;
}

static int do_read(int argc, char **argv) {
    if (argc != 5) { fprintf(stderr, "usage: sfa_tool read IN FRAME OUT\n"); return 2; }
    SFA *s = sfa_open(argv[2]);
    if (!s) { fprintf(stderr, "cannot open %s\n", argv[2]); return 1; }
    int frame = atoi(argv[3]);
    if (frame < 0) frame += (int)s->total_frames;
    if (frame < 0 || frame >= (int)s->total_frames) { fprintf(stderr, "frame out of range\n"); return 1; }
    uint8_t *buf = malloc(s->frame_bytes);
    if (!buf || sfa_read_frame(s, (uint32_t)frame, buf) != 0) { fprintf(stderr, "read failed\n"); return 1; }
    FILE *fp = fopen(argv[4], "wb");
    if (!fp) return 1;
    size_t n3 = (size_t)s->N_total;
    double *col = malloc(sizeof(double) * n3);
    uint64_t off = 0;
    for (uint32_t c = 0; c < s->n_columns; c++) {
        int dt = s->columns[c].dtype;
        const uint8_t *src = buf + off;
        for (size_t i = 0; i < n3; i++) {
            if (dt == SFA_F64) col[i] = ((const double *)src)[i];
            else if (dt == SFA_F32) col[i] = ((const float *)src)[i];
            else col[i] = sfa_f16_to_f32(((const uint16_t *)src)[i]);
        }
        fwrite(col, sizeof(double), n3, fp);
        printf("%s %d %d %d\n", s->columns[c].name, s->columns[c].semantic,
               s->columns[c].component, dt);
        off += n3 * sfa_dtype_size[dt];
    }
    fclose(fp);
    free(col);
    free(buf);
    sfa_close(s);
    return 0;
}

int main(int argc, char **argv) {
    if (argc >= 2 && !strcmp(argv[1], "write")) return do_write(argc, argv);
    if (argc >= 2 && !strcmp(argv[1], "read")) return do_read(argc, argv);
    fprintf(stderr, "usage: sfa_tool write|read ...\n");
    return 2;
}
