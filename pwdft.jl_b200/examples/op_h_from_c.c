/* A C host driving the hot path through include/pwb200.h alone, the way a
 * non-Python caller would bind the library.
 *
 * Builds the plane-wave basis of fcc Si (a = 10.2631 bohr, ecutwfc 15 Ha,
 * Gamma point) with the library's host functions, whose steps are those of
 * PWGrid.jl:79-92 (grid size), :199-242 (init_gvec) and :306-316
 * (init_gvecw). It then creates a context on device 0, sets a constant local
 * potential V0, and applies op_K + op_V_loc to a random block of host
 * ComplexF64 columns with pw_op_H_host. The result is checked against
 * 0.5 |G|^2 psi + V0 psi computed here; a constant potential acts as
 * multiplication in G space.
 *
 * Exit status: 0 on agreement (relative error < 1e-11), 1 on a mismatch,
 * 2 when the library reports an error such as "no CUDA device".
 *
 *   gcc -std=c99 -O2 -I../../include op_h_from_c.c -L../pwb200 -lpwb200 \
 *       -Wl,-rpath,'$ORIGIN/../pwb200' -lm -o op_h_from_c
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include "pwb200.h"

static int fail(pw_ctx *ctx, const char *what, int st) {
    fprintf(stderr, "%s failed (status %d): %s\n", what, st, ctx ? pw_last_error(ctx) : "no context");
    if (ctx) pw_destroy(ctx);
    return 2;
}

int main(void) {
    const double a = 10.2631, ecutwfc = 15.0, ecutrho = 4.0 * ecutwfc, V0 = -0.3;
    const double PI = 3.14159265358979323846;
    /* gen_lattice_fcc: columns a/2 (-1,0,1), a/2 (0,1,1), a/2 (-1,1,0) (column-major) */
    const double L[9] = {-0.5 * a, 0.0, 0.5 * a, 0.0, 0.5 * a, 0.5 * a, -0.5 * a, 0.5 * a, 0.0};
    /* RecVecs = 2 pi inv(LatVecs)^T, column-major */
    const double det = L[0] * (L[4] * L[8] - L[7] * L[5]) - L[3] * (L[1] * L[8] - L[7] * L[2]) +
                       L[6] * (L[1] * L[5] - L[4] * L[2]);
    double inv[9];
    inv[0] = (L[4] * L[8] - L[7] * L[5]) / det;
    inv[3] = -(L[3] * L[8] - L[6] * L[5]) / det;
    inv[6] = (L[3] * L[7] - L[6] * L[4]) / det;
    inv[1] = -(L[1] * L[8] - L[7] * L[2]) / det;
    inv[4] = (L[0] * L[8] - L[6] * L[2]) / det;
    inv[7] = -(L[0] * L[7] - L[6] * L[1]) / det;
    inv[2] = (L[1] * L[5] - L[4] * L[2]) / det;
    inv[5] = -(L[0] * L[5] - L[3] * L[2]) / det;
    inv[8] = (L[0] * L[4] - L[3] * L[1]) / det;
    double R[9];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) R[i + 3 * j] = 2.0 * PI * inv[j + 3 * i];
    int32_t Ns[3];
    for (int i = 0; i < 3; ++i) {
        const double len = sqrt(L[3 * i] * L[3 * i] + L[3 * i + 1] * L[3 * i + 1] + L[3 * i + 2] * L[3 * i + 2]);
        Ns[i] = pw_good_fft_order(2 * (int)lround(sqrt(ecutrho / 2.0) * len / PI) + 1);
    }
    int64_t Ng = 0;
    int st = pw_gvec_count(Ns, R, ecutrho, &Ng);
    if (st) return fail(NULL, "pw_gvec_count", st);
    double *G = malloc(sizeof(double) * 3 * Ng), *G2 = malloc(sizeof(double) * Ng), *Gk2 = malloc(sizeof(double) * Ng);
    int64_t *g2r = malloc(sizeof(int64_t) * Ng), *gw2g = malloc(sizeof(int64_t) * Ng), *gw2r = malloc(sizeof(int64_t) * Ng);
    if ((st = pw_gvec_build(Ns, R, ecutrho, Ng, G, G2, g2r))) return fail(NULL, "pw_gvec_build", st);
    const double k0[3] = {0.0, 0.0, 0.0};
    int64_t Ngw = 0;
    if ((st = pw_gvecw_build(Ng, G, g2r, k0, ecutwfc, &Ngw, gw2g, gw2r, Gk2))) return fail(NULL, "pw_gvecw_build", st);

    printf("basis: Ns = %d %d %d, Ng = %lld, Ngw = %lld\n", Ns[0], Ns[1], Ns[2], (long long)Ng, (long long)Ngw);
    fflush(stdout);
    const double vol = fabs(det);
    const int64_t *idx[1] = {gw2r};
    const double *gk2[1] = {Gk2};
    pw_grid_desc d = {{Ns[0], Ns[1], Ns[2]}, 1, 1, 0, vol, &Ngw, idx, gk2};
    pw_ctx *ctx = NULL;
    if ((st = pw_create(0, &d, &ctx))) return fail(ctx, "pw_create", st);
    const int64_t N = (int64_t)Ns[0] * Ns[1] * Ns[2];
    double *V = malloc(sizeof(double) * N);
    for (int64_t i = 0; i < N; ++i) V[i] = V0;
    if ((st = pw_set_vloc(ctx, V, 1))) return fail(ctx, "pw_set_vloc", st);

    const int nb = 4;
    double *psi = malloc(sizeof(double) * 2 * Ngw * nb), *Hpsi = malloc(sizeof(double) * 2 * Ngw * nb);
    srand(7);
    for (int64_t i = 0; i < 2 * Ngw * nb; ++i) psi[i] = (double)rand() / RAND_MAX - 0.5;
    if ((st = pw_op_H_host(ctx, 0, 0, psi, Hpsi, Ngw, nb, PW_OP_K | PW_OP_VLOC, PW_C128)))
        return fail(ctx, "pw_op_H_host", st);
    double err = 0.0, mx = 0.0;
    for (int b = 0; b < nb; ++b)
        for (int64_t g = 0; g < Ngw; ++g)
            for (int c = 0; c < 2; ++c) {
                const int64_t o = 2 * (b * Ngw + g) + c;
                const double ref = (0.5 * Gk2[g] + V0) * psi[o];
                err = fmax(err, fabs(Hpsi[o] - ref));
                mx = fmax(mx, fabs(ref));
            }
    printf("op_K + op_V_loc relative error %.3e\n", err / mx);
    pw_destroy(ctx);
    free(G); free(G2); free(Gk2); free(g2r); free(gw2g); free(gw2r); free(V); free(psi); free(Hpsi);
    return err < 1e-11 * mx ? 0 : 1;
}
