/* ring: C host driver of the ring test cases on the GPU library.
 *
 *   ring <n> <m> <nt> [--order P] [--limiter] [--strict] [--device]
 *        [--frames FILE] [--ctl FILE]
 *
 * Set-up of the reference's test_init(n, m) (tests/init.c:15-103): uniform
 * grid, time step 0.0125, IORD 3 unless --order is given, faded solid-body
 * ring flow of inner radius 1 and outer radius n/2.5 about the grid centre
 * (generators/src/genring2d.c:8-64, genringf2d.c:9-67), the same on every
 * level, w = 1 when m > 3 (the 3D "spiral"), and a Gaussian source of sigma 6
 * and cut-off radius n/8 centred n/4 right of the centre
 * (gengauss2d.c:6-33 / gengauss3d.c:6-39).  m = 3 is the 2D form.
 *
 * Stepping: by default through the reference-compatible smolar() with host
 * arrays and the driver's pointer exchange (tests/ring2d/test.c:87-106);
 * with --device the field stays on the GPU (mpdata_step) and only the frames
 * come back, by queued copies that overlap the next step (the whole field
 * once, at the end).  --limiter switches the nonoscillatory option on.
 *
 * Output (headless): --frames writes, per step 0..nt, the u, v and c planes
 * of level 1 as n*n floats each (the reference's ring2d.bin layout,
 * tests/ring2d/test.c:39-41,51-53); --ctl writes a GrADS descriptor for it;
 * --final writes the whole last field (n*n*m floats, the raw concentration
 * file the reference's 3D driver leaves, tests/init.c:241-300).
 * Each step prints "step <it> <probe>" like the reference 2D driver
 * (tests/ring2d/test.c:56-57).
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "mpdata_b200.h"

typedef float real;

static void ring_flow(int n, real* u, real* v)
{
    const int cx = n / 2, cy = n / 2;
    const real rmin = 1, rmax = n / 2.5f, dx = 1, dy = 1;
    for (int iy = 0; iy < n; iy++)
        for (int ix = 0; ix < n; ix++) {
            real x = (real)(ix - cx), y = (real)(iy - cy);
            real r = (real)sqrt(x * x + y * y);
            if (r >= rmin && r <= rmax) {  /* solid body inside the ring */
                u[ix + n * iy] = -y / rmin * dx;
                v[ix + n * iy] = x / rmin * dy;
            } else if (r > rmax) {         /* exponential fade outside it */
                u[ix + n * iy] = (real)(-y / rmin * dx * exp((rmax - r) * dx));
                v[ix + n * iy] = (real)(x / rmin * dy * exp((rmax - r) * dy));
            }
        }
}

static void gauss(int n, int m, real* c)
{
    const int cx = n / 2 + n / 4, cy = n / 2;
    const real sigma = 6.0f, radius = (real)(n / 8);
    const real s2 = sigma * sigma;
    if (m > 3) {
        const int cs = (int)radius; /* the 3D source is centred at z = n/8 */
        for (int is = 0; is < m; is++)
            for (int iy = 0; iy < n; iy++)
                for (int ix = 0; ix < n; ix++) {
                    int dx = ix - cx, dy = iy - cy, ds = is - cs;
                    real x2 = (real)(dx * dx), y2 = (real)(dy * dy), z2 = (real)(ds * ds);
                    if (sqrt(x2 + y2 + z2) <= radius)
                        c[ix + n * iy + n * n * is] =
                            (real)exp(-0.5 * (x2 / s2 + y2 / s2 + z2 / s2));
                }
    } else {
        for (int iy = 0; iy < n; iy++)
            for (int ix = 0; ix < n; ix++) {
                int dx = ix - cx, dy = iy - cy;
                real x2 = (real)(dx * dx), y2 = (real)(dy * dy);
                if (sqrt(x2 + y2) <= radius)
                    c[ix + n * iy] = (real)exp(-0.5 * (x2 / s2 + y2 / s2));
            }
        for (int is = 1; is < m; is++) memcpy(c + (size_t)n * n * is, c, sizeof(real) * n * n);
    }
}

static int usage(void)
{
    fprintf(stderr, "ring <n> <m> <nt> [--order P] [--limiter] [--strict] [--device] "
                    "[--frames FILE] [--ctl FILE] [--final FILE]\n");
    return 2;
}

#define CHECK(call)                                                                   \
    do {                                                                              \
        int rc_ = (call);                                                             \
        if (rc_) {                                                                    \
            fprintf(stderr, "%s failed (%d): %s\n", #call, rc_, mpdata_last_error()); \
            return 1;                                                                 \
        }                                                                             \
    } while (0)

int main(int argc, char** argv)
{
    if (argc < 4) return usage();
    const int n = atoi(argv[1]), m = atoi(argv[2]), nt = atoi(argv[3]);
    int order = 3, limiter = 0, strict = 0, device = 0;
    const char* frames = NULL;
    const char* ctl = NULL;
    const char* final_path = NULL;
    for (int a = 4; a < argc; a++) {
        if (!strcmp(argv[a], "--order") && a + 1 < argc) order = atoi(argv[++a]);
        else if (!strcmp(argv[a], "--limiter")) limiter = 1;
        else if (!strcmp(argv[a], "--strict")) strict = 1;
        else if (!strcmp(argv[a], "--device")) device = 1;
        else if (!strcmp(argv[a], "--frames") && a + 1 < argc) frames = argv[++a];
        else if (!strcmp(argv[a], "--ctl") && a + 1 < argc) ctl = argv[++a];
        else if (!strcmp(argv[a], "--final") && a + 1 < argc) final_path = argv[++a];
        else return usage();
    }
    if (n < 3 || m < 3 || nt < 0 || order < 1) return usage();
    const size_t n2 = (size_t)n * n, np = n2 * m;
    real* u = calloc(np, sizeof(real));
    real* v = calloc(np, sizeof(real));
    real* w = calloc(np, sizeof(real));
    real* c0 = calloc(np, sizeof(real));
    real* c1 = calloc(np, sizeof(real));
    real* dx = malloc(sizeof(real) * n);
    real* dy = malloc(sizeof(real) * n);
    real* ds = malloc(sizeof(real) * m);
    if (!u || !v || !w || !c0 || !c1 || !dx || !dy || !ds) return 1;
    for (int i = 0; i < n; i++) dx[i] = dy[i] = 1;
    for (int k = 0; k < m; k++) ds[k] = 1;
    ring_flow(n, u, v);
    for (int k = 1; k < m; k++) {
        memcpy(u + n2 * k, u, sizeof(real) * n2);
        memcpy(v + n2 * k, v, sizeof(real) * n2);
    }
    if (m > 3)
        for (size_t q = 0; q < np; q++) w[q] = 1.0f;
    gauss(n, m, c0);
    const real dt = 0.0125f;

    mpdata_options opt;
    mpdata_default_options(&opt);
    opt.limiter = limiter;
    opt.strict = strict;
    CHECK(mpdata_set_default_options(&opt));

    FILE* fp = frames ? fopen(frames, "wb") : NULL;
    if (frames && !fp) return 1;
    if (fp) {
        fwrite(u + n2, sizeof(real), n2, fp);
        fwrite(v + n2, sizeof(real), n2, fp);
        fwrite(c0 + n2, sizeof(real), n2, fp);
    }
    printf("step 0\n");
    mpdata_handle h = NULL;
    if (device) {
        CHECK(mpdata_create(&h, n, n, m, MPDATA_F32, order, &opt));
        CHECK(mpdata_set_velocity(h, dx, dy, ds, dt, u, u, v, v, w, w, MPDATA_HOST));
        CHECK(mpdata_set_field(h, c0, MPDATA_HOST));
    }
    const size_t probe = (size_t)(n / 2 + n / 4) + (size_t)n * (n / 2) + n2;
    real* last = c0;
    if (device) {
        /* Frames (level 1) leave the GPU by queued copies into two pinned
         * buffers: step it+1 and its frame copy are queued before frame it is
         * written, so the file output overlaps the GPU's work. */
        real* fb[2];
        int tk[2] = {-1, -1};
        fb[0] = (real*)mpdata_host_alloc(sizeof(real) * n2);
        fb[1] = (real*)mpdata_host_alloc(sizeof(real) * n2);
        if (!fb[0] || !fb[1]) return 1;
#define QUEUE_STEP(b)                                                      \
    do {                                                                   \
        CHECK(mpdata_step(h, 1));                                          \
        tk[b] = mpdata_get_planes(h, 1, 1, fb[b], MPDATA_HOST_ASYNC);      \
        if (tk[b] < 0) {                                                   \
            fprintf(stderr, "frame copy failed: %s\n", mpdata_last_error()); \
            return 1;                                                      \
        }                                                                  \
    } while (0)
        if (nt >= 1) QUEUE_STEP(1);
        for (int it = 1; it <= nt; it++) {
            const int b = it & 1;
            if (it < nt) QUEUE_STEP(b ^ 1);
            CHECK(mpdata_wait(h, tk[b]));
            if (fp) {
                fwrite(u + n2, sizeof(real), n2, fp);
                fwrite(v + n2, sizeof(real), n2, fp);
                fwrite(fb[b], sizeof(real), n2, fp);
            }
            printf("step %d %f\n", it, fb[b][probe - n2]);
        }
#undef QUEUE_STEP
        CHECK(mpdata_get_field(h, c1, MPDATA_HOST));
        last = c1;
        mpdata_host_free(fb[0]);
        mpdata_host_free(fb[1]);
    }
    for (int it = 1; !device && it <= nt; it++) {
        CHECK(smolar(n, n, m, dx, dy, ds, dt, u, u, v, v, w, w, &c0, &c1, DIVERGENT, order));
        if (fp) {
            fwrite(u + n2, sizeof(real), n2, fp);
            fwrite(v + n2, sizeof(real), n2, fp);
            fwrite(c1 + n2, sizeof(real), n2, fp);
        }
        printf("step %d %f\n", it, c1[probe]);
        last = c1;
        real* t = c0;
        c0 = c1;
        c1 = t;
    }
    if (fp) fclose(fp);
    if (final_path) {
        FILE* f = fopen(final_path, "wb");
        if (!f) return 1;
        fwrite(last, sizeof(real), np, f);
        fclose(f);
    }
    if (ctl) {
        FILE* f = fopen(ctl, "w");
        if (!f) return 1;
        fprintf(f, "DSET ^%s\nTITLE MPDATA ring case\nUNDEF -9.99e33\n", frames ? frames : "frames.bin");
        fprintf(f, "XDEF %d LINEAR 1 1\nYDEF %d LINEAR 1 1\nZDEF 1 LINEAR 1 1\n", n, n);
        fprintf(f, "TDEF %d LINEAR 00:00Z01jan2000 1mn\nVARS 3\n", nt + 1);
        fprintf(f, "u 0 99 x velocity\nv 0 99 y velocity\nc 0 99 concentration\nENDVARS\n");
        fclose(f);
    }
    if (h) mpdata_destroy(h);
    free(u); free(v); free(w); free(c0); free(c1); free(dx); free(dy); free(ds);
    return 0;
}
