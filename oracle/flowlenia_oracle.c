/*
 * Flow Lenia CPU oracle — TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference crate's CPU time step
 * (`CpuPropagator::step`, src/compute/propagator.rs:239-420, and
 * `CpuPropagator3D::step`, src/compute/propagator3d.rs:119-308), kept in the
 * reference's operation order so that it can serve as the parity checker for
 * the CUDA engine.  Only the test suite, the smoke check and the CPU-baseline
 * leg of the benchmark load this library; the product never links it.
 *
 * The same source is compiled twice: with -DORC_F64 every quantity is a
 * double (the FP64 twin used to state the error of f32 results), otherwise
 * every quantity is a float and arithmetic follows the reference statement by
 * statement.  Build with -ffp-contract=off so no multiply-add is fused (Rust
 * never contracts).
 *
 * The reference computes its convolution with the rustfft crate ("6.2", an
 * unpinned semver range: the reference ships no lockfile and no vendored
 * sources).  rustfft is a mixed-radix complex FFT with twiddles computed in
 * f64 and rounded to the element type; this file restates the published
 * algorithm as a Stockham autosort mixed-radix FFT (radices 4, 2, 3, 5 and a
 * direct DFT for other prime factors) with f64-computed twiddles.  Its
 * rounding differs from rustfft's butterflies at the 1e-7 relative level, so
 * parity with rustfft itself is pinned only by the reference's own FFT tests
 * (src/compute/fft.rs:492-787), which this oracle passes.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifdef ORC_F64
typedef double real;
#define R_EXP exp
#define R_SQRT sqrt
#define R_FLOOR floor
#define R_CEIL ceil
#define R_ROUND round
#define R_FABS fabs
#define R_POW pow
#define R_LIT(x) (x)
#define ORC_SYM(name) orc64_##name
#else
typedef float real;
#define R_EXP expf
#define R_SQRT sqrtf
#define R_FLOOR floorf
#define R_CEIL ceilf
#define R_ROUND roundf
#define R_FABS fabsf
#define R_POW powf
#define R_LIT(x) (x##f)
#define ORC_SYM(name) orc32_##name
#endif

/* Sources with |m| below this are skipped by the reintegration
 * (reintegration.rs:74-76, reintegration3d.rs:69-71).  A test-only build sets
 * it to 0 to show that the reference's mass drift comes from this skip. */
#ifndef ORC_MASS_SKIP
#define ORC_MASS_SKIP 1e-10
#endif

#define EXPORT __attribute__((visibility("default")))

static inline real r_max(real a, real b) { return (a != a) ? b : ((b != b) ? a : (a > b ? a : b)); }
static inline real r_min(real a, real b) { return (a != a) ? b : ((b != b) ? a : (a < b ? a : b)); }

/* Rust `f32 as i32`: saturating, NaN -> 0. */
static inline int r_to_i32(real v) {
    if (v != v) return 0;
    if (v >= (real)2147483647.0) return 2147483647;
    if (v <= (real)-2147483648.0) return (-2147483647 - 1);
    return (int)v;
}

/* ---------------------------------------------------------------------- */
/* Kernel construction: src/compute/kernel.rs:32-92, kernel3d.rs:32-90     */
/* ---------------------------------------------------------------------- */

/* rings: n_rings x (amplitude, distance, width).  Returns the side length
 * (2r+1) and writes side^dims values to out (out may be NULL to query). */
EXPORT int ORC_SYM(kernel_build)(int dims, real radius, int max_radius, int n_rings,
                                 const real* rings, real* out) {
    int actual_radius = (int)R_ROUND(radius * (real)max_radius);
    if (actual_radius < 0) actual_radius = 0;
    int size = actual_radius * 2 + 1;
    if (!out) return size;
    real center = (real)actual_radius;
    size_t total = (size_t)size * size * (dims == 3 ? size : 1);
    memset(out, 0, total * sizeof(real));
    real sum = R_LIT(0.0);
    int zs = dims == 3 ? size : 1;
    for (int z = 0; z < zs; ++z)
        for (int y = 0; y < size; ++y)
            for (int x = 0; x < size; ++x) {
                real dx = (real)x - center;
                real dy = (real)y - center;
                real dist;
                if (dims == 3) {
                    real dz = (real)z - center;
                    dist = R_SQRT(dx * dx + dy * dy + dz * dz);
                } else {
                    dist = R_SQRT(dx * dx + dy * dy);
                }
                real norm_dist = dist / (real)actual_radius;
                if (norm_dist > R_LIT(1.0)) continue;
                real value = R_LIT(0.0);
                for (int r = 0; r < n_rings; ++r) {
                    real amp = rings[3 * r + 0], dist_r = rings[3 * r + 1], w = rings[3 * r + 2];
                    real ring_dist = R_FABS(norm_dist - dist_r);
                    real bump = amp * R_EXP(-ring_dist * ring_dist / (R_LIT(2.0) * w * w));
                    value += bump;
                }
                out[((size_t)z * size + y) * size + x] = value;
                sum += value;
            }
    if (sum > R_LIT(0.0)) {
        real inv_sum = R_LIT(1.0) / sum;
        for (size_t i = 0; i < total; ++i) out[i] *= inv_sum;
    }
    return size;
}

/* Wrap-padding for circular convolution: kernel.rs:98-117, kernel3d.rs:103-133.
 * Later taps overwrite earlier ones when the kernel is wider than the grid. */
EXPORT void ORC_SYM(kernel_pad)(const real* kern, int size, int dims, int W, int H, int D, real* out) {
    memset(out, 0, (size_t)W * H * D * sizeof(real));
    int center = size / 2;
    int zs = dims == 3 ? size : 1;
    for (int kz = 0; kz < zs; ++kz)
        for (int ky = 0; ky < size; ++ky)
            for (int kx = 0; kx < size; ++kx) {
                int dx = kx - center, dy = ky - center;
                int tx = (dx + W) % W, ty = (dy + H) % H, tz = 0;
                if (dims == 3) {
                    int dz = kz - center;
                    tz = (dz + D) % D;
                }
                out[((size_t)tz * H + ty) * W + tx] = kern[((size_t)kz * size + ky) * size + kx];
            }
}

/* ---------------------------------------------------------------------- */
/* FFT (restatement of a mixed-radix complex FFT; see file header)        */
/* ---------------------------------------------------------------------- */

typedef struct { real re, im; } cpx;

static inline cpx c_mul(cpx a, cpx b) {
    /* num_complex Mul: (a.re*b.re - a.im*b.im, a.re*b.im + a.im*b.re) */
    cpx r;
    r.re = a.re * b.re - a.im * b.im;
    r.im = a.re * b.im + a.im * b.re;
    return r;
}
static inline cpx c_add(cpx a, cpx b) { cpx r = {a.re + b.re, a.im + b.im}; return r; }
static inline cpx c_sub(cpx a, cpx b) { cpx r = {a.re - b.re, a.im - b.im}; return r; }

typedef struct {
    int n;
    int nf;
    int fac[40];
    cpx* w;   /* w[t] = exp(-2 pi i t / n), computed in double */
} fft_plan;

static void plan_init(fft_plan* p, int n) {
    p->n = n;
    p->nf = 0;
    int m = n;
    while (m % 4 == 0) { p->fac[p->nf++] = 4; m /= 4; }
    while (m % 2 == 0) { p->fac[p->nf++] = 2; m /= 2; }
    while (m % 3 == 0) { p->fac[p->nf++] = 3; m /= 3; }
    while (m % 5 == 0) { p->fac[p->nf++] = 5; m /= 5; }
    for (int f = 7; m > 1; f += 2)
        while (m % f == 0) { p->fac[p->nf++] = f; m /= f; }
    p->w = (cpx*)malloc(sizeof(cpx) * (size_t)n);
    for (int t = 0; t < n; ++t) {
        double ang = -2.0 * M_PI * (double)t / (double)n;
        p->w[t].re = (real)cos(ang);
        p->w[t].im = (real)sin(ang);
    }
}
static void plan_free(fft_plan* p) { free(p->w); p->w = NULL; }

/* One length-n transform, Stockham autosort.  inverse != 0 uses conjugate
 * roots and applies no scaling (rustfft convention). */
static void fft_exec(const fft_plan* p, cpx* x, cpx* work, int inverse) {
    int n = p->n;
    if (n <= 1) return;
    cpx* src = x;
    cpx* dst = work;
    int ns = 1;
    real sgn = inverse ? R_LIT(-1.0) : R_LIT(1.0);
    cpx v[64];
    cpx vv[64];
    for (int s = 0; s < p->nf; ++s) {
        int rad = p->fac[s];
        int np = n / rad;
        int tstep = n / (ns * rad);
        for (int j = 0; j < np; ++j) {
            int k = j % ns;
            for (int q = 0; q < rad; ++q) {
                cpx a = src[j + q * np];
                if (q && k) {
                    cpx tw = p->w[(size_t)k * q * tstep];
                    tw.im *= sgn;
                    a = c_mul(a, tw);
                }
                v[q] = a;
            }
            if (rad == 2) {
                vv[0] = c_add(v[0], v[1]);
                vv[1] = c_sub(v[0], v[1]);
            } else if (rad == 4) {
                cpx t0 = c_add(v[0], v[2]);
                cpx t1 = c_sub(v[0], v[2]);
                cpx t2 = c_add(v[1], v[3]);
                cpx t3 = c_sub(v[1], v[3]);
                /* forward: multiply t3 by -i; inverse: by +i */
                cpx t3r;
                if (!inverse) { t3r.re = t3.im; t3r.im = -t3.re; }
                else { t3r.re = -t3.im; t3r.im = t3.re; }
                vv[0] = c_add(t0, t2);
                vv[2] = c_sub(t0, t2);
                vv[1] = c_add(t1, t3r);
                vv[3] = c_sub(t1, t3r);
            } else {
                int wstep = n / rad;
                for (int r = 0; r < rad; ++r) {
                    cpx acc = v[0];
                    for (int q = 1; q < rad; ++q) {
                        cpx tw = p->w[(size_t)((q * r) % rad) * wstep];
                        tw.im *= sgn;
                        acc = c_add(acc, c_mul(v[q], tw));
                    }
                    vv[r] = acc;
                }
            }
            int out0 = (j / ns) * ns * rad + k;
            for (int r = 0; r < rad; ++r) dst[out0 + r * ns] = vv[r];
        }
        ns *= rad;
        cpx* t = src; src = dst; dst = t;
    }
    if (src != x) memcpy(x, src, sizeof(cpx) * (size_t)n);
}

/* n-D complex FFT over a [D][H][W] array: x axis, then y, then z (forward);
 * z, y, x for the inverse (fft.rs:329-393, fft3d.rs:335-452). */
typedef struct {
    int W, H, D;
    fft_plan px, py, pz;
} fft3_plan;

static void fft3_init(fft3_plan* p, int W, int H, int D) {
    p->W = W; p->H = H; p->D = D;
    plan_init(&p->px, W);
    plan_init(&p->py, H);
    plan_init(&p->pz, D);
}
static void fft3_free(fft3_plan* p) { plan_free(&p->px); plan_free(&p->py); plan_free(&p->pz); }

static void axis_pass(const fft_plan* pl, cpx* data, int W, int H, int D, int axis, int inverse,
                      cpx* line, cpx* work) {
    size_t slice = (size_t)W * H;
    if (axis == 0) {
        for (int z = 0; z < D; ++z)
            for (int y = 0; y < H; ++y) fft_exec(pl, data + z * slice + (size_t)y * W, work, inverse);
    } else if (axis == 1) {
        for (int z = 0; z < D; ++z)
            for (int x = 0; x < W; ++x) {
                for (int y = 0; y < H; ++y) line[y] = data[z * slice + (size_t)y * W + x];
                fft_exec(pl, line, work, inverse);
                for (int y = 0; y < H; ++y) data[z * slice + (size_t)y * W + x] = line[y];
            }
    } else {
        for (int y = 0; y < H; ++y)
            for (int x = 0; x < W; ++x) {
                for (int z = 0; z < D; ++z) line[z] = data[z * slice + (size_t)y * W + x];
                fft_exec(pl, line, work, inverse);
                for (int z = 0; z < D; ++z) data[z * slice + (size_t)y * W + x] = line[z];
            }
    }
}

static void fft3_forward(const fft3_plan* p, cpx* data, cpx* line, cpx* work) {
    axis_pass(&p->px, data, p->W, p->H, p->D, 0, 0, line, work);
    if (p->H > 1) axis_pass(&p->py, data, p->W, p->H, p->D, 1, 0, line, work);
    if (p->D > 1) axis_pass(&p->pz, data, p->W, p->H, p->D, 2, 0, line, work);
}
static void fft3_inverse(const fft3_plan* p, cpx* data, cpx* line, cpx* work) {
    if (p->D > 1) axis_pass(&p->pz, data, p->W, p->H, p->D, 2, 1, line, work);
    if (p->H > 1) axis_pass(&p->py, data, p->W, p->H, p->D, 1, 1, line, work);
    axis_pass(&p->px, data, p->W, p->H, p->D, 0, 1, line, work);
}

static int max3(int a, int b, int c) { int m = a > b ? a : b; return m > c ? m : c; }

/* FftConvolver::fft2d / FftConvolver3D::fft3d: real in -> complex out (re/im planes). */
EXPORT void ORC_SYM(fft_forward)(const real* in, int W, int H, int D, real* out_re, real* out_im) {
    size_t N = (size_t)W * H * D;
    fft3_plan p;
    fft3_init(&p, W, H, D);
    cpx* data = (cpx*)malloc(sizeof(cpx) * N);
    int m = max3(W, H, D);
    cpx* line = (cpx*)malloc(sizeof(cpx) * (size_t)m);
    cpx* work = (cpx*)malloc(sizeof(cpx) * (size_t)m);
    for (size_t i = 0; i < N; ++i) { data[i].re = in[i]; data[i].im = R_LIT(0.0); }
    fft3_forward(&p, data, line, work);
    for (size_t i = 0; i < N; ++i) { out_re[i] = data[i].re; out_im[i] = data[i].im; }
    free(data); free(line); free(work);
    fft3_free(&p);
}

/* FftConvolver::ifft2d / ifft3d: complex in -> real part * 1/N out. */
EXPORT void ORC_SYM(fft_inverse)(const real* in_re, const real* in_im, int W, int H, int D, real* out) {
    size_t N = (size_t)W * H * D;
    fft3_plan p;
    fft3_init(&p, W, H, D);
    cpx* data = (cpx*)malloc(sizeof(cpx) * N);
    int m = max3(W, H, D);
    cpx* line = (cpx*)malloc(sizeof(cpx) * (size_t)m);
    cpx* work = (cpx*)malloc(sizeof(cpx) * (size_t)m);
    for (size_t i = 0; i < N; ++i) { data[i].re = in_re[i]; data[i].im = in_im[i]; }
    fft3_inverse(&p, data, line, work);
    real scale = R_LIT(1.0) / (real)(N);
    for (size_t i = 0; i < N; ++i) out[i] = data[i].re * scale;
    free(data); free(line); free(work);
    fft3_free(&p);
}

/* FftConvolver::convolve (fft.rs:162-176): both operands spatial. */
EXPORT void ORC_SYM(fft_convolve)(const real* in, const real* kern_padded, int W, int H, int D, real* out) {
    size_t N = (size_t)W * H * D;
    fft3_plan p;
    fft3_init(&p, W, H, D);
    cpx* a = (cpx*)malloc(sizeof(cpx) * N);
    cpx* b = (cpx*)malloc(sizeof(cpx) * N);
    int m = max3(W, H, D);
    cpx* line = (cpx*)malloc(sizeof(cpx) * (size_t)m);
    cpx* work = (cpx*)malloc(sizeof(cpx) * (size_t)m);
    for (size_t i = 0; i < N; ++i) {
        a[i].re = in[i]; a[i].im = R_LIT(0.0);
        b[i].re = kern_padded[i]; b[i].im = R_LIT(0.0);
    }
    fft3_forward(&p, a, line, work);
    fft3_forward(&p, b, line, work);
    for (size_t i = 0; i < N; ++i) a[i] = c_mul(a[i], b[i]);
    fft3_inverse(&p, a, line, work);
    real scale = R_LIT(1.0) / (real)(N);
    for (size_t i = 0; i < N; ++i) out[i] = a[i].re * scale;
    free(a); free(b); free(line); free(work);
    fft3_free(&p);
}

/* Direct circular convolution used by the reference's FFT-vs-direct test
 * (fft.rs:686-716): out[x] = sum_k in[x + k - r] * kern[k]. */
EXPORT void ORC_SYM(direct_convolve2d)(const real* in, const real* kern, int W, int H, int r, real* out) {
    int ks = 2 * r + 1;
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            real sum = R_LIT(0.0);
            for (int ky = 0; ky < ks; ++ky)
                for (int kx = 0; kx < ks; ++kx) {
                    int dx = kx - r, dy = ky - r;
                    int sx = ((x + dx + W) % W + W) % W;
                    int sy = ((y + dy + H) % H + H) % H;
                    sum += in[(size_t)sy * W + sx] * kern[(size_t)ky * ks + kx];
                }
            out[(size_t)y * W + x] = sum;
        }
}

/* ---------------------------------------------------------------------- */
/* Growth: src/compute/growth.rs:11-15, 45-59                              */
/* ---------------------------------------------------------------------- */

EXPORT real ORC_SYM(growth)(real u, real mu, real sigma) {
    real diff = u - mu;
    real sigma_sq_2 = R_LIT(2.0) * sigma * sigma;
    return R_LIT(2.0) * R_EXP(-diff * diff / sigma_sq_2) - R_LIT(1.0);
}

EXPORT void ORC_SYM(growth_accumulate)(const real* conv, real* target, size_t n, real weight, real mu,
                                       real sigma) {
    real sigma_sq_2 = R_LIT(2.0) * sigma * sigma;
    real inv_sigma_sq_2 = R_LIT(1.0) / sigma_sq_2;
    for (size_t i = 0; i < n; ++i) {
        real diff = conv[i] - mu;
        real g = R_LIT(2.0) * R_EXP(-diff * diff * inv_sigma_sq_2) - R_LIT(1.0);
        target[i] += weight * g;
    }
}

/* ---------------------------------------------------------------------- */
/* Sobel: gradient.rs:68-108, gradient3d.rs:41-147                         */
/* ---------------------------------------------------------------------- */

EXPORT void ORC_SYM(sobel2d)(const real* grid, real* gx_out, real* gy_out, int W, int H) {
    for (int y = 0; y < H; ++y) {
        int y_prev = (y + H - 1) % H, y_next = (y + 1) % H;
        size_t rp = (size_t)y_prev * W, rc = (size_t)y * W, rn = (size_t)y_next * W;
        for (int x = 0; x < W; ++x) {
            int x_prev = (x + W - 1) % W, x_next = (x + 1) % W;
            real tl = grid[rp + x_prev], tc = grid[rp + x], tr = grid[rp + x_next];
            real ml = grid[rc + x_prev], mr = grid[rc + x_next];
            real bl = grid[rn + x_prev], bc = grid[rn + x], br = grid[rn + x_next];
            real gx = (-tl + tr - R_LIT(2.0) * ml + R_LIT(2.0) * mr - bl + br) * R_LIT(0.125);
            real gy = (-tl - R_LIT(2.0) * tc - tr + bl + R_LIT(2.0) * bc + br) * R_LIT(0.125);
            gx_out[rc + x] = gx;
            gy_out[rc + x] = gy;
        }
    }
}

EXPORT void ORC_SYM(sobel3d)(const real* g, real* gx_out, real* gy_out, real* gz_out, int W, int H, int D) {
    size_t S = (size_t)W * H;
    for (int z = 0; z < D; ++z) {
        int zp = (z + D - 1) % D, zn = (z + 1) % D;
        for (int y = 0; y < H; ++y) {
            int yp = (y + H - 1) % H, yn = (y + 1) % H;
            for (int x = 0; x < W; ++x) {
                int xp = (x + W - 1) % W, xn = (x + 1) % W;
#define P(zz, yy, xx) g[(size_t)(zz) * S + (size_t)(yy) * W + (xx)]
                real p_mmm = P(zp, yp, xp), p_mm0 = P(zp, yp, x), p_mmp = P(zp, yp, xn);
                real p_m0m = P(zp, y, xp), p_m00 = P(zp, y, x), p_m0p = P(zp, y, xn);
                real p_mpm = P(zp, yn, xp), p_mp0 = P(zp, yn, x), p_mpp = P(zp, yn, xn);
                real p_0mm = P(z, yp, xp), p_0m0 = P(z, yp, x), p_0mp = P(z, yp, xn);
                real p_00m = P(z, y, xp), p_00p = P(z, y, xn);
                real p_0pm = P(z, yn, xp), p_0p0 = P(z, yn, x), p_0pp = P(z, yn, xn);
                real p_pmm = P(zn, yp, xp), p_pm0 = P(zn, yp, x), p_pmp = P(zn, yp, xn);
                real p_p0m = P(zn, y, xp), p_p00 = P(zn, y, x), p_p0p = P(zn, y, xn);
                real p_ppm = P(zn, yn, xp), p_pp0 = P(zn, yn, x), p_ppp = P(zn, yn, xn);
#undef P
                const real two = R_LIT(2.0);
                real gx_zm = -(p_mmm + two * p_m0m + p_mpm) + (p_mmp + two * p_m0p + p_mpp);
                real gx_z0 = -(p_0mm + two * p_00m + p_0pm) + (p_0mp + two * p_00p + p_0pp);
                real gx_zp = -(p_pmm + two * p_p0m + p_ppm) + (p_pmp + two * p_p0p + p_ppp);
                real gx = (gx_zm + two * gx_z0 + gx_zp) / R_LIT(32.0);
                real gy_zm = -(p_mmm + two * p_mm0 + p_mmp) + (p_mpm + two * p_mp0 + p_mpp);
                real gy_z0 = -(p_0mm + two * p_0m0 + p_0mp) + (p_0pm + two * p_0p0 + p_0pp);
                real gy_zp = -(p_pmm + two * p_pm0 + p_pmp) + (p_ppm + two * p_pp0 + p_ppp);
                real gy = (gy_zm + two * gy_z0 + gy_zp) / R_LIT(32.0);
                real gz_xm = -(p_mmm + two * p_m0m + p_mpm) + (p_pmm + two * p_p0m + p_ppm);
                real gz_x0 = -(p_mm0 + two * p_m00 + p_mp0) + (p_pm0 + two * p_p00 + p_pp0);
                real gz_xp = -(p_mmp + two * p_m0p + p_mpp) + (p_pmp + two * p_p0p + p_ppp);
                real gz = (gz_xm + two * gz_x0 + gz_xp) / R_LIT(32.0);
                size_t idx = (size_t)z * S + (size_t)y * W + x;
                gx_out[idx] = gx;
                gy_out[idx] = gy;
                gz_out[idx] = gz;
            }
        }
    }
}

/* ---------------------------------------------------------------------- */
/* Flow: flow.rs:14-32 (alpha), 68-87 (2D field), flow3d.rs:50-73          */
/* ---------------------------------------------------------------------- */

EXPORT real ORC_SYM(alpha)(real mass, real beta_a, real n) {
    real ratio = mass / beta_a;
    real powered;
    if (n == R_LIT(1.0)) powered = ratio;
    else if (n == R_LIT(2.0)) powered = ratio * ratio;
    else if (n == R_LIT(3.0)) powered = ratio * ratio * ratio;
    else if (n == R_LIT(4.0)) { real r2 = ratio * ratio; powered = r2 * r2; }
    else powered = R_POW(ratio, n);
    /* f32::clamp(0, 1): NaN passes through */
    if (powered < R_LIT(0.0)) powered = R_LIT(0.0);
    if (powered > R_LIT(1.0)) powered = R_LIT(1.0);
    return powered;
}

EXPORT void ORC_SYM(flow_field)(int dims, const real* gu, const real* ga, const real* mass_sum, size_t n,
                                real beta_a, real nexp, real* flow) {
    /* gu, ga, flow: dims planes of n values each (x, y[, z]) */
    for (size_t i = 0; i < n; ++i) {
        real alpha = ORC_SYM(alpha)(mass_sum[i], beta_a, nexp);
        real oma = R_LIT(1.0) - alpha;
        for (int d = 0; d < dims; ++d) flow[d * n + i] = oma * gu[d * n + i] - alpha * ga[d * n + i];
    }
}

/* ---------------------------------------------------------------------- */
/* Reintegration: reintegration.rs:60-174, reintegration3d.rs:56-198       */
/* ---------------------------------------------------------------------- */

EXPORT int ORC_SYM(wrap_coord)(int coord, int size) { return ((coord % size) + size) % size; }

static void distribute_mass_2d(real* grid, real mass, real dest_x, real dest_y, int W, int H, real s) {
    real x_min = dest_x - s, x_max = dest_x + s;
    real y_min = dest_y - s, y_max = dest_y + s;
    int ix_min = r_to_i32(R_FLOOR(x_min)); if (ix_min < -W) ix_min = -W;
    int ix_max = r_to_i32(R_CEIL(x_max));  if (ix_max > 2 * W) ix_max = 2 * W;
    int iy_min = r_to_i32(R_FLOOR(y_min)); if (iy_min < -H) iy_min = -H;
    int iy_max = r_to_i32(R_CEIL(y_max));  if (iy_max > 2 * H) iy_max = 2 * H;
    real total_area = (R_LIT(2.0) * s) * (R_LIT(2.0) * s);
    if (total_area < R_LIT(1e-10)) {
        int nx = ORC_SYM(wrap_coord)(r_to_i32(R_ROUND(dest_x)), W);
        int ny = ORC_SYM(wrap_coord)(r_to_i32(R_ROUND(dest_y)), H);
        grid[(size_t)ny * W + nx] += mass;
        return;
    }
    for (int iy = iy_min; iy <= iy_max; ++iy)
        for (int ix = ix_min; ix <= ix_max; ++ix) {
            real cx0 = (real)ix, cx1 = (real)(ix + 1);
            real cy0 = (real)iy, cy1 = (real)(iy + 1);
            real ox0 = r_max(cx0, x_min), ox1 = r_min(cx1, x_max);
            real oy0 = r_max(cy0, y_min), oy1 = r_min(cy1, y_max);
            real ow = r_max(ox1 - ox0, R_LIT(0.0));
            real oh = r_max(oy1 - oy0, R_LIT(0.0));
            real area = ow * oh;
            if (area > R_LIT(0.0)) {
                real fraction = area / total_area;
                real cell_mass = mass * fraction;
                int nx = ORC_SYM(wrap_coord)(ix, W);
                int ny = ORC_SYM(wrap_coord)(iy, H);
                grid[(size_t)ny * W + nx] += cell_mass;
            }
        }
}

/* `next` must be zeroed by the caller (propagator.rs:360). */
EXPORT void ORC_SYM(advect2d)(const real* cur, const real* fx, const real* fy, real* next, int W, int H,
                              real dt, real s) {
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            size_t idx = (size_t)y * W + x;
            real mass = cur[idx];
            if (R_FABS(mass) < (real)ORC_MASS_SKIP) continue;
            real dest_x = (real)x + dt * fx[idx];
            real dest_y = (real)y + dt * fy[idx];
            distribute_mass_2d(next, mass, dest_x, dest_y, W, H, s);
        }
}

static void distribute_mass_3d(real* grid, real mass, real dx_, real dy_, real dz_, int W, int H, int D,
                               real s) {
    real x_min = dx_ - s, x_max = dx_ + s;
    real y_min = dy_ - s, y_max = dy_ + s;
    real z_min = dz_ - s, z_max = dz_ + s;
    int ix_min = r_to_i32(R_FLOOR(x_min)); if (ix_min < -W) ix_min = -W;
    int ix_max = r_to_i32(R_CEIL(x_max));  if (ix_max > 2 * W) ix_max = 2 * W;
    int iy_min = r_to_i32(R_FLOOR(y_min)); if (iy_min < -H) iy_min = -H;
    int iy_max = r_to_i32(R_CEIL(y_max));  if (iy_max > 2 * H) iy_max = 2 * H;
    int iz_min = r_to_i32(R_FLOOR(z_min)); if (iz_min < -D) iz_min = -D;
    int iz_max = r_to_i32(R_CEIL(z_max));  if (iz_max > 2 * D) iz_max = 2 * D;
    real total_volume = (R_LIT(2.0) * s) * (R_LIT(2.0) * s) * (R_LIT(2.0) * s);
    size_t S = (size_t)W * H;
    if (total_volume < R_LIT(1e-10)) {
        int nx = ORC_SYM(wrap_coord)(r_to_i32(R_ROUND(dx_)), W);
        int ny = ORC_SYM(wrap_coord)(r_to_i32(R_ROUND(dy_)), H);
        int nz = ORC_SYM(wrap_coord)(r_to_i32(R_ROUND(dz_)), D);
        grid[(size_t)nz * S + (size_t)ny * W + nx] += mass;
        return;
    }
    for (int iz = iz_min; iz <= iz_max; ++iz)
        for (int iy = iy_min; iy <= iy_max; ++iy)
            for (int ix = ix_min; ix <= ix_max; ++ix) {
                real ox0 = r_max((real)ix, x_min), ox1 = r_min((real)(ix + 1), x_max);
                real oy0 = r_max((real)iy, y_min), oy1 = r_min((real)(iy + 1), y_max);
                real oz0 = r_max((real)iz, z_min), oz1 = r_min((real)(iz + 1), z_max);
                real ow = r_max(ox1 - ox0, R_LIT(0.0));
                real oh = r_max(oy1 - oy0, R_LIT(0.0));
                real od = r_max(oz1 - oz0, R_LIT(0.0));
                real vol = ow * oh * od;
                if (vol > R_LIT(0.0)) {
                    real fraction = vol / total_volume;
                    real cell_mass = mass * fraction;
                    int nx = ORC_SYM(wrap_coord)(ix, W);
                    int ny = ORC_SYM(wrap_coord)(iy, H);
                    int nz = ORC_SYM(wrap_coord)(iz, D);
                    grid[(size_t)nz * S + (size_t)ny * W + nx] += cell_mass;
                }
            }
}

EXPORT void ORC_SYM(advect3d)(const real* cur, const real* fx, const real* fy, const real* fz, real* next,
                              int W, int H, int D, real dt, real s) {
    size_t S = (size_t)W * H;
    for (int z = 0; z < D; ++z)
        for (int y = 0; y < H; ++y)
            for (int x = 0; x < W; ++x) {
                size_t idx = (size_t)z * S + (size_t)y * W + x;
                real mass = cur[idx];
                if (R_FABS(mass) < (real)ORC_MASS_SKIP) continue;
                real dest_x = (real)x + dt * fx[idx];
                real dest_y = (real)y + dt * fy[idx];
                real dest_z = (real)z + dt * fz[idx];
                distribute_mass_3d(next, mass, dest_x, dest_y, dest_z, W, H, D, s);
            }
}

/* naive f32 sum, reintegration.rs:221-228 */
EXPORT real ORC_SYM(total_mass)(const real* grid, size_t n) {
    real s = R_LIT(0.0);
    for (size_t i = 0; i < n; ++i) s += grid[i];
    return s;
}

/* ---------------------------------------------------------------------- */
/* Propagator: propagator.rs:157-420, propagator3d.rs:49-308               */
/* ---------------------------------------------------------------------- */

typedef struct {
    int W, H, D, C, K, dims;
    real dt, beta_a, nexp, s;
    int* src;
    int* tgt;
    real* weight;
    real* mu;
    real* sigma;
    cpx** khat;        /* K spectra, N bins each */
    fft3_plan plan;
    /* scratch */
    real** aff;
    real** next;
    real** conv;
    cpx** fscratch;    /* per kernel, N */
    cpx** line;        /* per kernel, max dim */
    cpx** work;        /* per kernel, max dim */
    real* csum;
    real* ga;          /* dims * N */
    real** gu;         /* per channel dims * N */
    real** flow;       /* per channel dims * N */
} orc_prop;

/* kparams: K x 6 (radius, weight, mu, sigma, source_channel, target_channel);
 * ring_count: K; rings: sum(ring_count) x 3 (amplitude, distance, width). */
EXPORT orc_prop* ORC_SYM(prop_new)(int W, int H, int D, int C, real dt, int kernel_radius, int K,
                                   const real* kparams, const int* ring_count, const real* rings,
                                   real beta_a, real nexp, real s) {
    orc_prop* p = (orc_prop*)calloc(1, sizeof(orc_prop));
    p->W = W; p->H = H; p->D = D; p->C = C; p->K = K;
    p->dims = D > 1 ? 3 : 2;
    p->dt = dt; p->beta_a = beta_a; p->nexp = nexp; p->s = s;
    size_t N = (size_t)W * H * D;
    int m = max3(W, H, D);
    fft3_init(&p->plan, W, H, D);
    p->src = (int*)malloc(sizeof(int) * (K > 0 ? K : 1));
    p->tgt = (int*)malloc(sizeof(int) * (K > 0 ? K : 1));
    p->weight = (real*)malloc(sizeof(real) * (K > 0 ? K : 1));
    p->mu = (real*)malloc(sizeof(real) * (K > 0 ? K : 1));
    p->sigma = (real*)malloc(sizeof(real) * (K > 0 ? K : 1));
    p->khat = (cpx**)calloc(K > 0 ? K : 1, sizeof(cpx*));
    p->conv = (real**)calloc(K > 0 ? K : 1, sizeof(real*));
    p->fscratch = (cpx**)calloc(K > 0 ? K : 1, sizeof(cpx*));
    p->line = (cpx**)calloc(K > 0 ? K : 1, sizeof(cpx*));
    p->work = (cpx**)calloc(K > 0 ? K : 1, sizeof(cpx*));
    int roff = 0;
    cpx* l0 = (cpx*)malloc(sizeof(cpx) * (size_t)m);
    cpx* w0 = (cpx*)malloc(sizeof(cpx) * (size_t)m);
    for (int k = 0; k < K; ++k) {
        const real* kp = kparams + 6 * k;
        p->weight[k] = kp[1]; p->mu[k] = kp[2]; p->sigma[k] = kp[3];
        p->src[k] = (int)kp[4]; p->tgt[k] = (int)kp[5];
        int size = ORC_SYM(kernel_build)(p->dims, kp[0], kernel_radius, ring_count[k], rings + 3 * roff, NULL);
        size_t ksz = (size_t)size * size * (p->dims == 3 ? size : 1);
        real* kern = (real*)malloc(sizeof(real) * ksz);
        ORC_SYM(kernel_build)(p->dims, kp[0], kernel_radius, ring_count[k], rings + 3 * roff, kern);
        roff += ring_count[k];
        real* padded = (real*)malloc(sizeof(real) * N);
        ORC_SYM(kernel_pad)(kern, size, p->dims, W, H, D, padded);
        p->khat[k] = (cpx*)malloc(sizeof(cpx) * N);
        for (size_t i = 0; i < N; ++i) { p->khat[k][i].re = padded[i]; p->khat[k][i].im = R_LIT(0.0); }
        fft3_forward(&p->plan, p->khat[k], l0, w0);
        free(padded);
        free(kern);
        p->conv[k] = (real*)malloc(sizeof(real) * N);
        p->fscratch[k] = (cpx*)malloc(sizeof(cpx) * N);
        p->line[k] = (cpx*)malloc(sizeof(cpx) * (size_t)m);
        p->work[k] = (cpx*)malloc(sizeof(cpx) * (size_t)m);
    }
    free(l0); free(w0);
    p->aff = (real**)calloc(C, sizeof(real*));
    p->next = (real**)calloc(C, sizeof(real*));
    p->gu = (real**)calloc(C, sizeof(real*));
    p->flow = (real**)calloc(C, sizeof(real*));
    for (int c = 0; c < C; ++c) {
        p->aff[c] = (real*)malloc(sizeof(real) * N);
        p->next[c] = (real*)malloc(sizeof(real) * N);
        p->gu[c] = (real*)malloc(sizeof(real) * N * p->dims);
        p->flow[c] = (real*)malloc(sizeof(real) * N * p->dims);
    }
    p->csum = (real*)malloc(sizeof(real) * N);
    p->ga = (real*)malloc(sizeof(real) * N * p->dims);
    return p;
}

EXPORT void ORC_SYM(prop_free)(orc_prop* p) {
    if (!p) return;
    for (int k = 0; k < p->K; ++k) {
        free(p->khat[k]); free(p->conv[k]); free(p->fscratch[k]); free(p->line[k]); free(p->work[k]);
    }
    for (int c = 0; c < p->C; ++c) { free(p->aff[c]); free(p->next[c]); free(p->gu[c]); free(p->flow[c]); }
    free(p->khat); free(p->conv); free(p->fscratch); free(p->line); free(p->work);
    free(p->aff); free(p->next); free(p->gu); free(p->flow);
    free(p->src); free(p->tgt); free(p->weight); free(p->mu); free(p->sigma);
    free(p->csum); free(p->ga);
    fft3_free(&p->plan);
    free(p);
}

/* Convolution (parallel over kernels) + growth accumulation in kernel order.
 * state: C planes of N values.  aff_out: C planes (may be NULL -> internal). */
static void prop_affinity(orc_prop* p, const real* state, int nthreads) {
    size_t N = (size_t)p->W * p->H * p->D;
    for (int c = 0; c < p->C; ++c) memset(p->aff[c], 0, sizeof(real) * N);
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads) if (nthreads > 1)
    for (int k = 0; k < p->K; ++k) {
        cpx* f = p->fscratch[k];
        const real* srcp = state + (size_t)p->src[k] * N;
        for (size_t i = 0; i < N; ++i) { f[i].re = srcp[i]; f[i].im = R_LIT(0.0); }
        fft3_forward(&p->plan, f, p->line[k], p->work[k]);
        for (size_t i = 0; i < N; ++i) f[i] = c_mul(f[i], p->khat[k][i]);
        fft3_inverse(&p->plan, f, p->line[k], p->work[k]);
        real scale = R_LIT(1.0) / (real)(N);
        for (size_t i = 0; i < N; ++i) p->conv[k][i] = f[i].re * scale;
    }
    for (int k = 0; k < p->K; ++k)
        ORC_SYM(growth_accumulate)(p->conv[k], p->aff[p->tgt[k]], N, p->weight[k], p->mu[k], p->sigma[k]);
}

/* Mass sum, gradients, flow and reintegration (parallel over channels). */
static void prop_transport(orc_prop* p, const real* state, real* const* aff, real* out, int nthreads) {
    size_t N = (size_t)p->W * p->H * p->D;
    memset(p->csum, 0, sizeof(real) * N);
    for (int c = 0; c < p->C; ++c) {
        const real* ch = state + (size_t)c * N;
        for (size_t i = 0; i < N; ++i) p->csum[i] += ch[i];
    }
    if (p->dims == 2) ORC_SYM(sobel2d)(p->csum, p->ga, p->ga + N, p->W, p->H);
    else ORC_SYM(sobel3d)(p->csum, p->ga, p->ga + N, p->ga + 2 * N, p->W, p->H, p->D);
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads) if (nthreads > 1)
    for (int c = 0; c < p->C; ++c) {
        if (p->dims == 2) ORC_SYM(sobel2d)(aff[c], p->gu[c], p->gu[c] + N, p->W, p->H);
        else ORC_SYM(sobel3d)(aff[c], p->gu[c], p->gu[c] + N, p->gu[c] + 2 * N, p->W, p->H, p->D);
        ORC_SYM(flow_field)(p->dims, p->gu[c], p->ga, p->csum, N, p->beta_a, p->nexp, p->flow[c]);
        memset(p->next[c], 0, sizeof(real) * N);
        const real* cur = state + (size_t)c * N;
        if (p->dims == 2)
            ORC_SYM(advect2d)(cur, p->flow[c], p->flow[c] + N, p->next[c], p->W, p->H, p->dt, p->s);
        else
            ORC_SYM(advect3d)(cur, p->flow[c], p->flow[c] + N, p->flow[c] + 2 * N, p->next[c], p->W, p->H, p->D,
                              p->dt, p->s);
    }
    for (int c = 0; c < p->C; ++c) memcpy(out + (size_t)c * N, p->next[c], sizeof(real) * N);
}

/* Advance `state` (C planes of N values, in place) by `steps` steps. */
EXPORT void ORC_SYM(prop_run)(orc_prop* p, real* state, int steps, int nthreads) {
    for (int t = 0; t < steps; ++t) {
        prop_affinity(p, state, nthreads);
        prop_transport(p, state, p->aff, state, nthreads);
    }
}

/* Stage entry points for stage-level parity tests. */
EXPORT void ORC_SYM(prop_affinity)(orc_prop* p, const real* state, real* aff_out) {
    size_t N = (size_t)p->W * p->H * p->D;
    prop_affinity(p, state, 1);
    for (int c = 0; c < p->C; ++c) memcpy(aff_out + (size_t)c * N, p->aff[c], sizeof(real) * N);
}

EXPORT void ORC_SYM(prop_transport)(orc_prop* p, const real* state, const real* aff, real* out) {
    size_t N = (size_t)p->W * p->H * p->D;
    real** a = (real**)malloc(sizeof(real*) * p->C);
    for (int c = 0; c < p->C; ++c) a[c] = (real*)(aff + (size_t)c * N);
    prop_transport(p, state, a, out, 1);
    free(a);
}

/* Flow field per channel (dims planes each) after a transport stage. */
EXPORT void ORC_SYM(prop_last_flow)(orc_prop* p, real* flow_out) {
    size_t N = (size_t)p->W * p->H * p->D;
    for (int c = 0; c < p->C; ++c) memcpy(flow_out + (size_t)c * N * p->dims, p->flow[c], sizeof(real) * N * p->dims);
}

/* Many independent worlds, parallel over worlds (evolution/search.rs:152-172). */
EXPORT void ORC_SYM(prop_run_many)(orc_prop** props, real** states, int n_worlds, int steps, int nthreads) {
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads) if (nthreads > 1)
    for (int w = 0; w < n_worlds; ++w) ORC_SYM(prop_run)(props[w], states[w], steps, 1);
}

/* ---------------------------------------------------------------------- */
/* EmbeddedPropagator: per-cell parameters advected with mass              */
/* (src/compute/embedded_propagator.rs:222-372, direct_convolution.rs:     */
/* 129-177, param_advection.rs:83-165 and 263-320, schema/embedding.rs:    */
/* 64-166).  CellParams are 5 consecutive reals per cell, in the order of  */
/* the struct (embedding.rs:20-31): mu, sigma, weight, beta_a, n.          */
/* ---------------------------------------------------------------------- */

#define NPAR 5

/* CellParams::default (embedding.rs:33-43) */
static const real cell_default[NPAR] = {R_LIT(0.15), R_LIT(0.015), R_LIT(1.0), R_LIT(1.0), R_LIT(2.0)};

/* convolve_growth_accumulate_embedded (direct_convolution.rs:133-177):
 * correlation sum in ky-major order skipping zero taps, then the growth with
 * the cell's own mu/sigma/weight (of the target channel). */
EXPORT void ORC_SYM(conv_growth_acc_embedded)(const real* input, const real* kern, int ksize, const real* params,
                                              real* target, int W, int H) {
    int k_half = ksize / 2;
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            size_t idx = (size_t)y * W + x;
            real conv_sum = R_LIT(0.0);
            for (int ky = 0; ky < ksize; ++ky)
                for (int kx = 0; kx < ksize; ++kx) {
                    real k_val = kern[ky * ksize + kx];
                    if (k_val == R_LIT(0.0)) continue;
                    int sx = ORC_SYM(wrap_coord)(x + kx - k_half, W);
                    int sy = ORC_SYM(wrap_coord)(y + ky - k_half, H);
                    conv_sum += input[(size_t)sy * W + sx] * k_val;
                }
            const real* cp = params + NPAR * idx;
            real diff = conv_sum - cp[0];
            real sigma_sq_2 = R_LIT(2.0) * cp[1] * cp[1];
            real g = R_LIT(2.0) * R_EXP(-diff * diff / sigma_sq_2) - R_LIT(1.0);
            target[idx] += cp[2] * g;
        }
}

/* compute_distribution_overlap (param_advection.rs:263-300) */
EXPORT real ORC_SYM(distribution_overlap)(real dest_x, real dest_y, real s, real cell_x, real cell_y) {
    real dist_x_min = dest_x - s, dist_x_max = dest_x + s;
    real dist_y_min = dest_y - s, dist_y_max = dest_y + s;
    real cell_x_max = cell_x + R_LIT(1.0), cell_y_max = cell_y + R_LIT(1.0);
    real ox0 = r_max(dist_x_min, cell_x), ox1 = r_min(dist_x_max, cell_x_max);
    real oy0 = r_max(dist_y_min, cell_y), oy1 = r_min(dist_y_max, cell_y_max);
    real ow = r_max(ox1 - ox0, R_LIT(0.0));
    real oh = r_max(oy1 - oy0, R_LIT(0.0));
    real area = ow * oh;
    real total_area = (R_LIT(2.0) * s) * (R_LIT(2.0) * s);
    if (total_area > R_LIT(1e-10)) return area / total_area;
    return (cell_x <= dest_x && dest_x < cell_x_max && cell_y <= dest_y && dest_y < cell_y_max) ? R_LIT(1.0)
                                                                                                : R_LIT(0.0);
}

/* CellParams::mix_softmax (embedding.rs:64-125): masses[i] with params rows
 * prm[i] (NPAR each). */
EXPORT void ORC_SYM(mix_softmax)(const real* masses, const real* const* prm, int n, real temperature,
                                 real* out) {
    if (n == 0) { memcpy(out, cell_default, sizeof(cell_default)); return; }
    if (n == 1) { memcpy(out, prm[0], sizeof(real) * NPAR); return; }
    real max_mass = -(real)INFINITY;
    for (int i = 0; i < n; ++i) max_mass = r_max(max_mass, masses[i]);
    real* w = (real*)malloc(sizeof(real) * (size_t)n);
    real weight_sum = R_LIT(0.0);
    for (int i = 0; i < n; ++i) {
        w[i] = R_EXP((masses[i] - max_mass) / temperature);
        weight_sum += w[i];
    }
    if (weight_sum > R_LIT(0.0)) {
        for (int i = 0; i < n; ++i) w[i] /= weight_sum;
    } else {
        real uniform = R_LIT(1.0) / (real)n;
        for (int i = 0; i < n; ++i) w[i] = uniform;
    }
    for (int f = 0; f < NPAR; ++f) out[f] = R_LIT(0.0);
    for (int i = 0; i < n; ++i)
        for (int f = 0; f < NPAR; ++f) out[f] += prm[i][f] * w[i];
    free(w);
}

/* CellParams::mix_linear (embedding.rs:127-166) */
EXPORT void ORC_SYM(mix_linear)(const real* masses, const real* const* prm, int n, real* out) {
    if (n == 0) { memcpy(out, cell_default, sizeof(cell_default)); return; }
    if (n == 1) { memcpy(out, prm[0], sizeof(real) * NPAR); return; }
    real total = R_LIT(0.0);
    for (int i = 0; i < n; ++i) total += masses[i];
    if (total <= R_LIT(0.0)) { memcpy(out, cell_default, sizeof(cell_default)); return; }
    for (int f = 0; f < NPAR; ++f) out[f] = R_LIT(0.0);
    for (int i = 0; i < n; ++i) {
        real w = masses[i] / total;
        for (int f = 0; f < NPAR; ++f) out[f] += prm[i][f] * w;
    }
}

/* compute_max_flow_magnitude (param_advection.rs:303-309): fold(0, f32::max). */
EXPORT real ORC_SYM(max_flow_magnitude)(const real* fx, const real* fy, size_t n) {
    real m = R_LIT(0.0);
    for (size_t i = 0; i < n; ++i) m = r_max(m, R_SQRT(fx[i] * fx[i] + fy[i] * fy[i]));
    return m;
}

/* advect_mass_and_params_into (param_advection.rs:83-165), a gather over
 * (2R+1)^2 wrapped offsets in dy-major order with R from the largest flow
 * magnitude.  The overlap is taken between the source's square placed at its
 * wrapped index plus dt*F and the unwrapped destination cell, as the
 * reference does.  next_params is left untouched where no mass arrives. */
EXPORT void ORC_SYM(advect_params2d)(const real* mass, const real* params, const real* fx, const real* fy,
                                     int linear, real temperature, real dt, real s, int W, int H, real* next_mass,
                                     real* next_params) {
    real max_flow = ORC_SYM(max_flow_magnitude)(fx, fy, (size_t)W * H);
    int R = r_to_i32(R_CEIL(max_flow * dt + s)) + 1;
    int cap = (2 * R + 1) * (2 * R + 1);
    real* cm = (real*)malloc(sizeof(real) * (size_t)cap);
    const real** cpp = (const real**)malloc(sizeof(real*) * (size_t)cap);
    for (int dest_y = 0; dest_y < H; ++dest_y)
        for (int dest_x = 0; dest_x < W; ++dest_x) {
            size_t dest_idx = (size_t)dest_y * W + dest_x;
            int n = 0;
            real total_mass = R_LIT(0.0);
            for (int dy = -R; dy <= R; ++dy)
                for (int dx = -R; dx <= R; ++dx) {
                    int src_x = ORC_SYM(wrap_coord)(dest_x + dx, W);
                    int src_y = ORC_SYM(wrap_coord)(dest_y + dy, H);
                    size_t src_idx = (size_t)src_y * W + src_x;
                    real src_mass = mass[src_idx];
                    if (R_FABS(src_mass) < R_LIT(1e-10)) continue;
                    real dest_fx = (real)src_x + dt * fx[src_idx];
                    real dest_fy = (real)src_y + dt * fy[src_idx];
                    real overlap = ORC_SYM(distribution_overlap)(dest_fx, dest_fy, s, (real)dest_x, (real)dest_y);
                    if (overlap > R_LIT(0.0)) {
                        real mc = src_mass * overlap;
                        total_mass += mc;
                        cm[n] = mc;
                        cpp[n] = params + NPAR * src_idx;
                        ++n;
                    }
                }
            next_mass[dest_idx] = total_mass;
            if (n > 0 && total_mass > R_LIT(1e-10)) {
                real* out = next_params + NPAR * dest_idx;
                if (n == 1) memcpy(out, cpp[0], sizeof(real) * NPAR);
                else if (linear) ORC_SYM(mix_linear)(cm, cpp, n, out);
                else ORC_SYM(mix_softmax)(cm, cpp, n, temperature, out);
            }
        }
    free(cm);
    free(cpp);
}

typedef struct {
    int W, H, C, K;
    real dt, s, temperature;
    int enabled, linear;
    int* src;
    int* tgt;
    int* ksize;
    real** kern;
    real** aff;
    real** next;
    real* next_params;  /* C x N x NPAR: the propagator's own parameter buffer */
    real* csum;
    real* ga;           /* 2 x N */
    real* gu;           /* 2 x N */
    real* flow;         /* 2 x N */
} orc_emb;

/* EmbeddedPropagator::new (embedded_propagator.rs:177-221).  kparams: K x 6
 * (radius, weight, mu, sigma, source_channel, target_channel) as for
 * prop_new; only the stencils and channels are used (growth takes the cells'
 * parameters).  The propagator's next parameter buffer starts at
 * CellParams::default(). */
EXPORT orc_emb* ORC_SYM(emb_new)(int W, int H, int C, real dt, int kernel_radius, int K, const real* kparams,
                                 const int* ring_count, const real* rings, real s, int enabled, int linear,
                                 real temperature) {
    orc_emb* p = (orc_emb*)calloc(1, sizeof(orc_emb));
    p->W = W; p->H = H; p->C = C; p->K = K;
    p->dt = dt; p->s = s; p->enabled = enabled; p->linear = linear; p->temperature = temperature;
    size_t N = (size_t)W * H;
    int kk = K > 0 ? K : 1;
    p->src = (int*)malloc(sizeof(int) * kk);
    p->tgt = (int*)malloc(sizeof(int) * kk);
    p->ksize = (int*)malloc(sizeof(int) * kk);
    p->kern = (real**)calloc(kk, sizeof(real*));
    int roff = 0;
    for (int k = 0; k < K; ++k) {
        const real* kp = kparams + 6 * k;
        p->src[k] = (int)kp[4];
        p->tgt[k] = (int)kp[5];
        int size = ORC_SYM(kernel_build)(2, kp[0], kernel_radius, ring_count[k], rings + 3 * roff, NULL);
        p->ksize[k] = size;
        p->kern[k] = (real*)malloc(sizeof(real) * (size_t)size * size);
        ORC_SYM(kernel_build)(2, kp[0], kernel_radius, ring_count[k], rings + 3 * roff, p->kern[k]);
        roff += ring_count[k];
    }
    p->aff = (real**)calloc(C, sizeof(real*));
    p->next = (real**)calloc(C, sizeof(real*));
    for (int c = 0; c < C; ++c) {
        p->aff[c] = (real*)malloc(sizeof(real) * N);
        p->next[c] = (real*)malloc(sizeof(real) * N);
    }
    p->next_params = (real*)malloc(sizeof(real) * N * C * NPAR);
    for (size_t i = 0; i < N * C; ++i) memcpy(p->next_params + NPAR * i, cell_default, sizeof(cell_default));
    p->csum = (real*)malloc(sizeof(real) * N);
    p->ga = (real*)malloc(sizeof(real) * 2 * N);
    p->gu = (real*)malloc(sizeof(real) * 2 * N);
    p->flow = (real*)malloc(sizeof(real) * 2 * N);
    return p;
}

EXPORT void ORC_SYM(emb_free)(orc_emb* p) {
    if (!p) return;
    for (int k = 0; k < p->K; ++k) free(p->kern[k]);
    for (int c = 0; c < p->C; ++c) { free(p->aff[c]); free(p->next[c]); }
    free(p->kern); free(p->src); free(p->tgt); free(p->ksize);
    free(p->aff); free(p->next); free(p->next_params);
    free(p->csum); free(p->ga); free(p->gu); free(p->flow);
    free(p);
}

/* The propagator's own parameter buffer (C x N x NPAR), for checks of the
 * buffer-swap semantics. */
EXPORT void ORC_SYM(emb_next_params)(orc_emb* p, real* out) {
    memcpy(out, p->next_params, sizeof(real) * (size_t)p->W * p->H * p->C * NPAR);
}

/* EmbeddedPropagator::step (embedded_propagator.rs:222-339) on
 * state[C][N] and params[C][N][NPAR], in place: channels and parameter grids
 * are swapped with the propagator's buffers as the reference swaps them. */
EXPORT void ORC_SYM(emb_step)(orc_emb* p, real* state, real* params, int steps) {
    size_t N = (size_t)p->W * p->H;
    size_t PN = N * NPAR;
    for (int t = 0; t < steps; ++t) {
        for (int c = 0; c < p->C; ++c) memset(p->aff[c], 0, sizeof(real) * N);
        for (int k = 0; k < p->K; ++k)
            ORC_SYM(conv_growth_acc_embedded)(state + (size_t)p->src[k] * N, p->kern[k], p->ksize[k],
                                              params + (size_t)p->tgt[k] * PN, p->aff[p->tgt[k]], p->W, p->H);
        memset(p->csum, 0, sizeof(real) * N);
        for (int c = 0; c < p->C; ++c)
            for (size_t i = 0; i < N; ++i) p->csum[i] += state[(size_t)c * N + i];
        ORC_SYM(sobel2d)(p->csum, p->ga, p->ga + N, p->W, p->H);
        for (int c = 0; c < p->C; ++c) {
            const real* cp = params + (size_t)c * PN;
            ORC_SYM(sobel2d)(p->aff[c], p->gu, p->gu + N, p->W, p->H);
            /* compute_flow_field_embedded_into (embedded_propagator.rs:353-372) */
            for (size_t i = 0; i < N; ++i) {
                real alpha = ORC_SYM(alpha)(p->csum[i], cp[NPAR * i + 3], cp[NPAR * i + 4]);
                real oma = R_LIT(1.0) - alpha;
                p->flow[i] = oma * p->gu[i] - alpha * p->ga[i];
                p->flow[N + i] = oma * p->gu[N + i] - alpha * p->ga[N + i];
            }
            real* np_c = p->next_params + (size_t)c * PN;
            if (p->enabled) {
                ORC_SYM(advect_params2d)(state + (size_t)c * N, cp, p->flow, p->flow + N, p->linear,
                                         p->temperature, p->dt, p->s, p->W, p->H, p->next[c], np_c);
            } else {
                memset(p->next[c], 0, sizeof(real) * N);
                ORC_SYM(advect2d)(state + (size_t)c * N, p->flow, p->flow + N, p->next[c], p->W, p->H, p->dt,
                                  p->s);
                memcpy(np_c, cp, sizeof(real) * PN);
            }
        }
        /* swap channels (contents) and parameter grids with the propagator's buffers */
        for (int c = 0; c < p->C; ++c) {
            real* cur = state + (size_t)c * N;
            for (size_t i = 0; i < N; ++i) { real v = cur[i]; cur[i] = p->next[c][i]; p->next[c][i] = v; }
        }
        for (size_t i = 0; i < PN * p->C; ++i) {
            real v = params[i]; params[i] = p->next_params[i]; p->next_params[i] = v;
        }
    }
}

/* ---------------------------------------------------------------------- */
/* Seeds: src/schema/seed.rs:160-524                                       */
/* grid: C x D x H x W, accumulated in place.                              */
/* ---------------------------------------------------------------------- */

static void gauss2d(real* grid, int W, int H, real cx, real cy, real radius, real amp) {
    real sigma_sq = (radius / R_LIT(2.0)) * (radius / R_LIT(2.0));
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            real dx = (real)x - cx, dy = (real)y - cy;
            real dist_sq = dx * dx + dy * dy;
            grid[(size_t)y * W + x] += amp * R_EXP(-dist_sq / (R_LIT(2.0) * sigma_sq));
        }
}

static void gauss3d(real* grid, int W, int H, int D, real cx, real cy, real cz, real radius, real amp) {
    real sigma_sq = (radius / R_LIT(2.0)) * (radius / R_LIT(2.0));
    for (int z = 0; z < D; ++z)
        for (int y = 0; y < H; ++y)
            for (int x = 0; x < W; ++x) {
                real dx = (real)x - cx, dy = (real)y - cy, dz = (real)z - cz;
                real dist_sq = dx * dx + dy * dy + dz * dz;
                grid[((size_t)z * H + y) * W + x] += amp * R_EXP(-dist_sq / (R_LIT(2.0) * sigma_sq));
            }
}

static void ring2d(real* grid, int W, int H, real cx, real cy, real r_in, real r_out, real amp) {
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            real dx = (real)x - cx, dy = (real)y - cy;
            real dist = R_SQRT(dx * dx + dy * dy);
            if (dist >= r_in && dist <= r_out) {
                real edge = (r_out - r_in) * R_LIT(0.2);
                real inner = r_min((dist - r_in) / edge, R_LIT(1.0));
                real outer = r_min((r_out - dist) / edge, R_LIT(1.0));
                grid[(size_t)y * W + x] += amp * r_min(inner, outer);
            }
        }
}

static void shell3d(real* grid, int W, int H, int D, real cx, real cy, real cz, real r_in, real r_out,
                    real amp) {
    for (int z = 0; z < D; ++z)
        for (int y = 0; y < H; ++y)
            for (int x = 0; x < W; ++x) {
                real dx = (real)x - cx, dy = (real)y - cy, dz = (real)z - cz;
                real dist = R_SQRT(dx * dx + dy * dy + dz * dz);
                if (dist >= r_in && dist <= r_out) {
                    real edge = (r_out - r_in) * R_LIT(0.2);
                    real inner = r_min((dist - r_in) / edge, R_LIT(1.0));
                    real outer = r_min((r_out - dist) / edge, R_LIT(1.0));
                    grid[((size_t)z * H + y) * W + x] += amp * r_min(inner, outer);
                }
            }
}

static void torus3d(real* grid, int W, int H, int D, real cx, real cy, real cz, real rmaj, real rmin,
                    real amp) {
    real sigma_sq = (rmin / R_LIT(2.0)) * (rmin / R_LIT(2.0));
    for (int z = 0; z < D; ++z)
        for (int y = 0; y < H; ++y)
            for (int x = 0; x < W; ++x) {
                real dx = (real)x - cx, dy = (real)y - cy, dz = (real)z - cz;
                real dist_xy = R_SQRT(dx * dx + dy * dy);
                real ring_dx = dist_xy - rmaj;
                real dt_ = R_SQRT(ring_dx * ring_dx + dz * dz);
                real value = amp * R_EXP(-dt_ * dt_ / (R_LIT(2.0) * sigma_sq));
                if (value > R_LIT(1e-6)) grid[((size_t)z * H + y) * W + x] += value;
            }
}

/* kind: 0 GaussianBlob, 1 Ring, 2 GaussianSphere, 3 Shell, 4 Torus3D, 5 Noise.
 * f: pattern floats (center x,y[,z], then radii / amplitude as listed in
 * seed.rs); channel < 0 means "all channels" for Noise. */
EXPORT void ORC_SYM(seed_apply)(real* grid, int W, int H, int D, int C, int kind, const real* f, int channel,
                                uint64_t noise_seed) {
    size_t N = (size_t)W * H * D;
    int mn_xy = W < H ? W : H;
    int mn = mn_xy < D ? mn_xy : D;
    if (kind == 5) {
        uint64_t st = noise_seed;
        int c0 = channel < 0 ? 0 : channel, c1 = channel < 0 ? C : channel + 1;
        for (int c = c0; c < c1; ++c) {
            if (c >= C) continue;
            for (size_t i = 0; i < N; ++i) {
                st = st * 6364136223846793005ULL + 1ULL;
                real v = (real)(st >> 33) / (real)(1ULL << 31);
                grid[(size_t)c * N + i] += f[0] * v;
            }
        }
        return;
    }
    if (channel < 0 || channel >= C) return;
    real* g = grid + (size_t)channel * N;
    real cx = f[0] * (real)W, cy = f[1] * (real)H;
    if (kind == 0) {
        real r = f[2] * (real)mn_xy;
        if (D == 1) gauss2d(g, W, H, cx, cy, r, f[3]);
        else gauss3d(g, W, H, D, cx, cy, R_LIT(0.5) * (real)D, r, f[3]);
    } else if (kind == 1) {
        real r_in = f[2] * (real)mn_xy, r_out = f[3] * (real)mn_xy;
        if (D == 1) ring2d(g, W, H, cx, cy, r_in, r_out, f[4]);
        else shell3d(g, W, H, D, cx, cy, R_LIT(0.5) * (real)D, r_in, r_out, f[4]);
    } else {
        real cz = f[2] * (real)D;
        if (kind == 2) gauss3d(g, W, H, D, cx, cy, cz, f[3] * (real)mn, f[4]);
        else if (kind == 3) shell3d(g, W, H, D, cx, cy, cz, f[3] * (real)mn, f[4] * (real)mn, f[5]);
        else if (kind == 4) torus3d(g, W, H, D, cx, cy, cz, f[3] * (real)mn, f[4] * (real)mn, f[5]);
    }
}
