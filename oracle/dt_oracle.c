/*
 * CPU oracle for the disptools displacement-field generator.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is a plain-C restatement of the
 * reference algorithm (m-pilia/disptools v0.4.1, the C99 library under src/),
 * written to check the CUDA implementation in disptools_b200.  Only the test
 * suite, the smoke check and the CPU-baseline leg of the benchmark load it;
 * the product never links, loads or calls it.
 *
 * Parity is pinned: tests/test_oracle.py compares every function here with
 * the reference library compiled from its own sources (oracle/_ref, built by
 * oracle/Makefile) and with the committed golden vectors in tests/golden/.
 *
 * Layout conventions follow the reference (src/headers/disptools.h:30-36):
 * vector fields are [3][nz][ny][nx] (component-major, x fastest), scalar
 * maps are [nz][ny][nx], masks are C `bool`.
 *
 * The arithmetic is FP64 (FLOAT_SIZE=64 in the reference).  ORACLE_ORDER_PD
 * selects the interior finite-difference order (4 is the reference default,
 * CMakeLists.txt:99-104; 2 is used to check the analytic gradient).
 */
#include <float.h>
#include <math.h>
#include <stdbool.h>
#include <stddef.h>
#include <stdlib.h>
#include <string.h>

#ifndef ORACLE_REAL
#define ORACLE_REAL double
#endif
#ifndef ORACLE_ORDER_PD
#define ORACLE_ORDER_PD 4
#endif

typedef ORACLE_REAL real;

/* Finite-difference schemes along one axis.  The coefficients are those of
 * src/headers/jacobian_macros.h: one-sided second order (:7-99), central
 * second order (:101-119) and central fourth order (:121-148). */
enum { S_FWD = 0, S_BWD = 1, S_C2 = 2, S_C4 = 3 };

static const double K_TWO_THIRDS = 0.666666666666666666666666666;
static const double K_ONE_TWELFTH = 0.083333333333333333333333333;

typedef struct {
    size_t n[3];   /* nx, ny, nz */
    size_t N;      /* voxels */
    size_t st[3];  /* strides of x, y, z */
    real ih[3];    /* inverse spacing */
} grid_t;

static grid_t make_grid(size_t nx, size_t ny, size_t nz, real dx, real dy, real dz)
{
    grid_t g;
    g.n[0] = nx; g.n[1] = ny; g.n[2] = nz;
    g.N = nx * ny * nz;
    g.st[0] = 1; g.st[1] = nx; g.st[2] = nx * ny;
    /* src/jacobian.c:73-75 */
    g.ih[0] = 1.0 / dx; g.ih[1] = 1.0 / dy; g.ih[2] = 1.0 / dz;
    return g;
}

/* One partial derivative of a scalar component `c` (pointer at the voxel)
 * along an axis of stride `s`, with scheme `k` and inverse spacing `ih`. */
static inline double fd(const real *c, ptrdiff_t s, int k, real ih)
{
    switch (k) {
    case S_FWD: return (-1.5 * c[0] + 2.0 * c[s] - 0.5 * c[2 * s]) * ih;
    case S_BWD: return (+1.5 * c[0] - 2.0 * c[-s] + 0.5 * c[-2 * s]) * ih;
    case S_C2:  return (c[s] - c[-s]) * ih * .5;
    default:    return ((c[s] - c[-s]) * K_TWO_THIRDS - (c[2 * s] - c[-2 * s]) * K_ONE_TWELFTH) * ih;
    }
}

/* det(I + A), expanded along the first row as det3 in
 * src/headers/disptools.h:185-199. */
static inline double det_i_plus(const double a[3][3])
{
    const double a11 = a[0][0] + 1.0, a12 = a[0][1], a13 = a[0][2];
    const double a21 = a[1][0], a22 = a[1][1] + 1.0, a23 = a[1][2];
    const double a31 = a[2][0], a32 = a[2][1], a33 = a[2][2] + 1.0;
    return a11 * (a22 * a33 - a23 * a32)
         - a12 * (a21 * a33 - a23 * a31)
         + a13 * (a21 * a32 - a22 * a31);
}

/* Scheme used along each axis at voxel p.  This is the case analysis of
 * src/jacobian.c:70-242 stated per voxel instead of per region:
 *  - a voxel with any coordinate on the outer layer (0 or n-1) uses the
 *    one-sided second-order scheme along those axes (forward at 0, backward
 *    at n-1) and the central second-order scheme along the others
 *    (corners :117-141, edges :143-200, faces :175-220);
 *  - otherwise, with ORDER_PD == 4, a voxel with any coordinate on the
 *    penultimate layer (1 or n-2) uses the central second-order scheme on all
 *    axes (:223-241), and every other voxel the central fourth-order scheme
 *    (:87-110);
 *  - with ORDER_PD == 2 every non-boundary voxel is central second order. */
static inline void schemes_at(const grid_t *g, const size_t p[3], int k[3])
{
    bool outer = false, penult = false;
    for (int a = 0; a < 3; ++a) {
        if (p[a] == 0 || p[a] == g->n[a] - 1) outer = true;
        else if (p[a] == 1 || p[a] == g->n[a] - 2) penult = true;
    }
    for (int a = 0; a < 3; ++a) {
        if (outer) {
            k[a] = p[a] == 0 ? S_FWD : (p[a] == g->n[a] - 1 ? S_BWD : S_C2);
        } else if (ORACLE_ORDER_PD == 2 || penult) {
            k[a] = S_C2;
        } else {
            k[a] = S_C4;
        }
    }
}

static inline real jacobian_at(const grid_t *g, const real *f, const size_t p[3])
{
    int k[3];
    schemes_at(g, p, k);
    const size_t o = p[2] * g->st[2] + p[1] * g->st[1] + p[0];
    double a[3][3];
    for (int c = 0; c < 3; ++c)
        for (int ax = 0; ax < 3; ++ax)
            a[c][ax] = fd(f + c * g->N + o, (ptrdiff_t) g->st[ax], k[ax], g->ih[ax]);
    return (real) det_i_plus(a);
}

/* a1/a2: src/jacobian.c:7-21 (jacobian_dynamic) and :70-242 (jacobian). */
void oracle_jacobian(size_t nx, size_t ny, size_t nz, real dx, real dy, real dz,
                     const real *f, real *J)
{
    const grid_t g = make_grid(nx, ny, nz, dx, dy, dz);
    #pragma omp parallel for collapse(2) schedule(static)
    for (size_t z = 0; z < nz; ++z)
        for (size_t y = 0; y < ny; ++y)
            for (size_t x = 0; x < nx; ++x) {
                const size_t p[3] = {x, y, z};
                J[(z * ny + y) * nx + x] = jacobian_at(&g, f, p);
            }
}

/* src/jacobian.c:29-55 */
void oracle_regularise(size_t nx, size_t ny, size_t nz, real *J, real epsilon)
{
    const size_t N = nx * ny * nz;
    #pragma omp parallel for schedule(static)
    for (size_t i = 0; i < N; ++i)
        if (J[i] < epsilon) J[i] = epsilon;
}

/* a3: src/headers/error.h:87-172.  Writes the per-voxel error and returns
 * the total squared error; *max_error is the maximum |v| inside the mask. */
real oracle_compute_error(size_t N, const real *Jt, const real *Jf, const bool *mask,
                          real tolerance, real *v, real *max_error)
{
    real total = 0.0, mx = 0.0;
    #pragma omp parallel for schedule(static) reduction(+ : total) reduction(max : mx)
    for (size_t i = 0; i < N; ++i) {
        const real e = Jf[i] - Jt[i];
        real w;
        if (mask[i]) {
            w = e;
        } else {
            const real ae = fabs(e);
            w = ae < tolerance ? 0.0 : copysign(ae - tolerance, e);
        }
        v[i] = w;
        total += w * w;
        if (mask[i] && fabs(w) > mx) mx = fabs(w);
    }
    *max_error = mx;
    return total;
}

/* Second-order central-difference matrix I + grad(u) at voxel offset o,
 * the dfx_dx..dfz_dz macros of src/displacement_field_gradient.c:13-21.
 * Column `skip` is not evaluated (set to 0): the cofactors taken at the
 * neighbour p -/+ e_k never use the k column, and at p next to the boundary
 * its differences would read outside the volume. */
static inline void m2_at(const grid_t *g, const real *f, size_t o, int skip, double m[3][3])
{
    for (int c = 0; c < 3; ++c)
        for (int ax = 0; ax < 3; ++ax) {
            if (ax == skip) {
                m[c][ax] = 0.0;
                continue;
            }
            const real *q = f + c * g->N + o;
            const ptrdiff_t s = (ptrdiff_t) g->st[ax];
            m[c][ax] = (q[s] - q[-s]) * g->ih[ax] * .5 + (c == ax ? 1.0 : 0.0);
        }
}

/* The 2x2 minor of m that excludes row i and column k, with the factor order
 * used by the cofactor expressions of src/displacement_field_gradient.c:91-133. */
static inline double minor2(const double m[3][3], int i, int k)
{
    const int r0 = i == 0 ? 1 : 0, r1 = i == 2 ? 1 : 2;
    const int c0 = k == 0 ? 1 : 0, c1 = k == 2 ? 1 : 2;
    return m[r0][c0] * m[r1][c1] - m[r0][c1] * m[r1][c0];
}

/* a4: src/displacement_field_gradient.c:26-145.  Gradient of the cost with
 * respect to the field at the interior voxels; boundary voxels of g are left
 * untouched (the reference allocates g with calloc and never writes them). */
void oracle_gradient(size_t nx, size_t ny, size_t nz, real dx, real dy, real dz,
                     const real *f, const real *Jf, const real *v, real delta, real zeta,
                     real *gout, real *g_norm_2)
{
    const grid_t g = make_grid(nx, ny, nz, dx, dy, dz);
    real sq = 0.0;
    #pragma omp parallel for collapse(2) schedule(static) reduction(+ : sq)
    for (size_t z = 1; z < nz - 1; ++z)
        for (size_t y = 1; y < ny - 1; ++y)
            for (size_t x = 1; x < nx - 1; ++x) {
                const size_t o = (z * ny + y) * nx + x;
                double t[3][3];   /* t[i][k]: direction-k term of component i */
                for (int k = 0; k < 3; ++k) {
                    const size_t ob = o - g.st[k], of = o + g.st[k];
                    /* regularised errors at the two neighbours (:63-88) */
                    real eb = v[ob], ef = v[of];
                    if (Jf[ob] < delta) eb += zeta * (Jf[ob] - delta);
                    if (Jf[of] < delta) ef += zeta * (Jf[of] - delta);
                    double mb[3][3], mf[3][3];
                    m2_at(&g, f, ob, k, mb);
                    m2_at(&g, f, of, k, mf);
                    for (int i = 0; i < 3; ++i)
                        t[i][k] = g.ih[k] * (+eb * minor2(mb, i, k) - ef * minor2(mf, i, k));
                }
                /* cofactor signs (-1)^(i+k), summed in the order x, y, z */
                const real gx = (real) (t[0][0] - t[0][1] + t[0][2]);
                const real gy = (real) (-t[1][0] + t[1][1] - t[1][2]);
                const real gz = (real) (t[2][0] - t[2][1] + t[2][2]);
                gout[o] = gx;
                gout[g.N + o] = gy;
                gout[2 * g.N + o] = gz;
                sq += gx * gx + gy * gy + gz * gz;
            }
    *g_norm_2 = sq;
}

/* a5: src/displacement_field_gradient.c:150-175 */
static void move_field(size_t N, const real *old_f, real *new_f, const real *gr, real eta)
{
    #pragma omp parallel for schedule(static)
    for (size_t i = 0; i < 3 * N; ++i) new_f[i] = old_f[i] - eta * gr[i];
}

/* Run statistics returned by the oracle drivers (the reference drivers
 * return void and only print these when verbose). */
typedef struct {
    long iterations;      /* value of the loop counter when the loop ended */
    long trials;          /* candidate evaluations (jacobian + error) */
    long gradients;       /* gradient evaluations */
    int reason;           /* see ORACLE_STOP_* */
    double error;         /* total error of the returned field */
    double max_error;     /* masked max |v| of the returned field */
    double cand_error;    /* total error of the last evaluated candidate */
    double cand_max_error;
    double eta;           /* final step length */
} oracle_stats;

enum {
    ORACLE_STOP_IT_MAX = 0,
    ORACLE_STOP_ERROR_EXPLODED = 1,
    ORACLE_STOP_ETA = 2,
    ORACLE_STOP_THETA = 3,
    ORACLE_STOP_MAX_EXPLODED = 4,
    ORACLE_STOP_EPSILON = 5,
    ORACLE_STOP_ALLOC = 6,
};

/* a6: src/displacement_field_gradient.c:191-431 */
int oracle_generate_gradient(
    size_t nx, size_t ny, size_t nz, real dx, real dy, real dz,
    const real *Jt, const bool *mask,
    real epsilon, real tolerance, real eta, real eta_max, real alpha, real beta,
    real gamma, real delta, real zeta, real theta, real iota, bool strict,
    size_t it_max, real *field, oracle_stats *st)
{
    const size_t N = nx * ny * nz;
    real *fb[2], *jb[2];
    fb[0] = calloc(3 * N, sizeof(real));
    fb[1] = calloc(3 * N, sizeof(real));
    jb[0] = calloc(N, sizeof(real));
    jb[1] = calloc(N, sizeof(real));
    real *v = calloc(N, sizeof(real));
    real *gr = calloc(3 * N, sizeof(real));
    oracle_stats s = {0};
    if (!fb[0] || !fb[1] || !jb[0] || !jb[1] || !v || !gr) {
        s.reason = ORACLE_STOP_ALLOC;
        goto out;
    }
    int old_b = 0, new_b = 1;
    memcpy(fb[old_b], field, 3 * N * sizeof(real));

    /* initial error (:261-269) and gradient (:279-287) */
    real max_e, last_max = DBL_MAX, gn2;
    oracle_jacobian(nx, ny, nz, dx, dy, dz, fb[old_b], jb[old_b]);
    real last_e = oracle_compute_error(N, Jt, jb[old_b], mask, tolerance, v, &max_e);
    const real e0 = last_e, m0 = max_e;
    s.error = e0; s.max_error = m0;
    oracle_gradient(nx, ny, nz, dx, dy, dz, fb[old_b], jb[old_b], v, delta, zeta, gr, &gn2);
    s.gradients++;

    /* search for a large initial step (:289-317) */
    real err;
    do {
        eta *= alpha;
        move_field(N, fb[old_b], fb[new_b], gr, eta);
        oracle_jacobian(nx, ny, nz, dx, dy, dz, fb[new_b], jb[new_b]);
        err = oracle_compute_error(N, Jt, jb[new_b], mask, tolerance, v, &max_e);
        s.trials++;
    } while (eta < eta_max && err - last_e > -gamma * eta * gn2);
    eta /= alpha * alpha;

    /* restore the error of the initial field (:319-326) */
    last_e = oracle_compute_error(N, Jt, jb[old_b], mask, tolerance, v, &max_e);

    size_t it;
    s.reason = ORACLE_STOP_IT_MAX;
    for (it = 1; it <= it_max; ++it) {
        oracle_gradient(nx, ny, nz, dx, dy, dz, fb[old_b], jb[old_b], v, delta, zeta, gr, &gn2);
        s.gradients++;
        eta *= alpha;
        eta = eta > eta_max ? eta_max : eta;
        for (;;) {   /* backtracking (:344-375) */
            move_field(N, fb[old_b], fb[new_b], gr, eta);
            oracle_jacobian(nx, ny, nz, dx, dy, dz, fb[new_b], jb[new_b]);
            err = oracle_compute_error(N, Jt, jb[new_b], mask, tolerance, v, &max_e);
            s.trials++;
            const bool eta_good = eta >= iota;
            const bool ag = err - last_e > -gamma * eta * gn2;
            const bool sc = strict && max_e > last_max;
            if (eta_good && (ag || sc)) eta *= beta;
            else break;
        }
        s.cand_error = err; s.cand_max_error = max_e;
        /* stopping conditions (:387-410) */
        if (!isnormal(err)) { s.reason = ORACLE_STOP_ERROR_EXPLODED; break; }
        if (eta < iota) { s.reason = ORACLE_STOP_ETA; break; }
        if (1.0 - err / last_e < theta) { s.reason = ORACLE_STOP_THETA; break; }
        if (!isnormal(max_e)) { s.reason = ORACLE_STOP_MAX_EXPLODED; break; }
        if (max_e < epsilon) { s.reason = ORACLE_STOP_EPSILON; break; }
        last_e = err;
        last_max = max_e;
        s.error = err; s.max_error = max_e;
        int t = old_b; old_b = new_b; new_b = t;
    }
    s.iterations = (long) it;
    s.eta = eta;
    (void) e0; (void) m0;
    /* the last accepted field is returned (:421) */
    memcpy(field, fb[old_b], 3 * N * sizeof(real));
out:
    free(fb[0]); free(fb[1]); free(jb[0]); free(jb[1]); free(v); free(gr);
    if (st) *st = s;
    return s.reason == ORACLE_STOP_ALLOC ? -1 : 0;
}

/* a7: src/displacement_field_greedy.c:23-67.  Only interior voxels of the new
 * field are written; its boundary keeps whatever the buffer held. */
static void greedy_step(const grid_t *g, const real *old_f, real *new_f, const real *v,
                        real eta, real dx, real dy, real dz)
{
    const real ddx = eta * dx * .5f, ddy = eta * dy * .5f, ddz = eta * dz * .5f;
    const size_t nx = g->n[0], ny = g->n[1], nz = g->n[2], N = g->N;
    #pragma omp parallel for collapse(2) schedule(static)
    for (size_t z = 1; z < nz - 1; ++z)
        for (size_t y = 1; y < ny - 1; ++y)
            for (size_t x = 1; x < nx - 1; ++x) {
                const size_t o = (z * ny + y) * nx + x;
                const real ux = ddx * (v[o + 1] - v[o - 1]);
                const real uy = ddy * (v[o + nx] - v[o - nx]);
                const real uz = ddz * (v[o + nx * ny] - v[o - nx * ny]);
                new_f[o] = old_f[o] + ux;
                new_f[N + o] = old_f[N + o] + uy;
                new_f[2 * N + o] = old_f[2 * N + o] + uz;
            }
}

/* src/displacement_field_greedy.c:85-247 */
int oracle_generate_greedy(
    size_t nx, size_t ny, size_t nz, real dx, real dy, real dz,
    const real *Jt, const bool *mask,
    real epsilon, real tolerance, real eta, real eta_max, real alpha, real beta,
    real gamma, real delta, real zeta, real theta, real iota, bool strict,
    size_t it_max, real *field, oracle_stats *st)
{
    (void) eta_max; (void) alpha; (void) gamma; (void) delta; (void) zeta; (void) strict;
    const grid_t g = make_grid(nx, ny, nz, dx, dy, dz);
    const size_t N = g.N;
    real *fb[2], *jb[2];
    fb[0] = calloc(3 * N, sizeof(real));
    fb[1] = calloc(3 * N, sizeof(real));
    jb[0] = calloc(N, sizeof(real));
    jb[1] = calloc(N, sizeof(real));
    real *v = calloc(N, sizeof(real));
    oracle_stats s = {0};
    if (!fb[0] || !fb[1] || !jb[0] || !jb[1] || !v) {
        s.reason = ORACLE_STOP_ALLOC;
        goto out;
    }
    int old_b = 0, new_b = 1;
    memcpy(fb[old_b], field, 3 * N * sizeof(real));
    real max_e;
    oracle_jacobian(nx, ny, nz, dx, dy, dz, fb[old_b], jb[old_b]);
    real last_e = oracle_compute_error(N, Jt, jb[old_b], mask, tolerance, v, &max_e);
    s.error = last_e; s.max_error = max_e;
    size_t it;
    s.reason = ORACLE_STOP_IT_MAX;
    for (it = 1; it <= it_max; ++it) {
        greedy_step(&g, fb[old_b], fb[new_b], v, eta, dx, dy, dz);
        oracle_jacobian(nx, ny, nz, dx, dy, dz, fb[new_b], jb[new_b]);
        const real err = oracle_compute_error(N, Jt, jb[new_b], mask, tolerance, v, &max_e);
        s.trials++;
        s.cand_error = err; s.cand_max_error = max_e;
        if (!isnormal(err)) { s.reason = ORACLE_STOP_ERROR_EXPLODED; break; }
        if (err >= last_e) {   /* reject, shrink the step, repeat (:198-213) */
            eta *= beta;
            if (eta < iota) { s.reason = ORACLE_STOP_ETA; break; }
            --it;
            continue;
        }
        if (1.0 - err / last_e < theta) { s.reason = ORACLE_STOP_THETA; break; }
        if (!isnormal(max_e)) { s.reason = ORACLE_STOP_MAX_EXPLODED; break; }
        if (max_e < epsilon) { s.reason = ORACLE_STOP_EPSILON; break; }
        last_e = err;
        s.error = err; s.max_error = max_e;
        int t = old_b; old_b = new_b; new_b = t;
    }
    s.iterations = (long) it;
    s.eta = eta;
    memcpy(field, fb[old_b], 3 * N * sizeof(real));
out:
    free(fb[0]); free(fb[1]); free(jb[0]); free(jb[1]); free(v);
    if (st) *st = s;
    return s.reason == ORACLE_STOP_ALLOC ? -1 : 0;
}

int oracle_float_size(void) { return (int) (8 * sizeof(real)); }
int oracle_order_pd(void) { return ORACLE_ORDER_PD; }

/* One finite difference (scheme S_FWD=0, S_BWD=1, S_C2=2, S_C4=3) of a
 * component array at element `o` along stride `s`: the macros of
 * src/headers/jacobian_macros.h:7-148, exported to re-express the known
 * answers of test/c/test_jacobian_macros.cpp:70-148. */
double oracle_fd(const real *c, size_t o, size_t s, int k, real ih)
{
    return fd(c + o, (ptrdiff_t) s, k, ih);
}
