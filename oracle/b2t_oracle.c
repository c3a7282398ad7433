/*
 * b2t_oracle.c -- FP64 CPU restatement of the ASTRA CUDA projection model.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA library in
 * astra-toolbox_b200/csrc: only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference legs of bench.py load it.  Nothing in the product
 * path links, calls or falls back to it.
 *
 * Every function restates, in double precision and in plain loops, the sampling
 * model of one reference kernel (file:line cited at each function, paths
 * relative to the astra-toolbox source tree).  The model is the one the
 * reference's texture hardware evaluates:
 *   - linear filtering with texel centres at integer + 0.5 and a zero border
 *     (cuda/3d/util3d.cu:379-399, cuda/2d/util.cu:155-226);
 *   - an optional "tex8" mode that quantises the fractional interpolation
 *     weights to 1/256 the way the texture unit does (the reference's own 2D
 *     test emulates it the same way: tests/python/functional/test_line2d.py:14-16).
 *
 * Geometry is passed as the reference's per-view vector structs, unchanged:
 *   3D: 12 doubles per view, SConeProjection / SPar3DProjection layout
 *       (include/astra/GeometryUtil3D.h:47-115): src-or-ray xyz, detS xyz,
 *       detU xyz, detV xyz.
 *   2D: 6 floats per view, SFanProjection / SParProjection layout
 *       (include/astra/GeometryUtil2D.h:53-105).
 *
 * Array layouts follow the reference: volume [z][y][x], projections
 * [v][angle][u]; 2D volume [row][col], sinogram [angle][det].
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* ------------------------------------------------------------------------- */
/* thread helper                                                              */
/* ------------------------------------------------------------------------- */

typedef void (*orc_range_fn)(void *ctx, long begin, long end);

typedef struct {
    orc_range_fn fn;
    void *ctx;
    long begin, end;
} orc_job;

static void *orc_thread_main(void *p)
{
    orc_job *j = (orc_job *)p;
    j->fn(j->ctx, j->begin, j->end);
    return NULL;
}

/* Split [0, n) into nthreads contiguous pieces and run fn on each. */
static void orc_parallel(orc_range_fn fn, void *ctx, long n, int nthreads)
{
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    if ((long)nthreads > n) nthreads = (int)(n > 0 ? n : 1);
    if (nthreads == 1) {
        fn(ctx, 0, n);
        return;
    }
    pthread_t th[256];
    orc_job jobs[256];
    for (int t = 0; t < nthreads; ++t) {
        jobs[t].fn = fn;
        jobs[t].ctx = ctx;
        jobs[t].begin = n * t / nthreads;
        jobs[t].end = n * (t + 1) / nthreads;
        pthread_create(&th[t], NULL, orc_thread_main, &jobs[t]);
    }
    for (int t = 0; t < nthreads; ++t) pthread_join(th[t], NULL);
}

/* ------------------------------------------------------------------------- */
/* interpolation                                                              */
/* ------------------------------------------------------------------------- */

/* Texture-unit fractional weight: exact, or quantised to 8 fractional bits. */
static inline double orc_frac_weight(double a, int tex8)
{
    if (tex8) return nearbyint(a * 256.0) / 256.0;
    return a;
}

/*
 * Linear interpolation of a 2D plane at continuous index (q1, q2), where texel
 * (i1, i2) sits at q = (i1, i2).  Texels outside [0,n1) x [0,n2) read as zero
 * (cudaAddressModeBorder).  Element (i1, i2) lives at base[i1*s1 + i2*s2].
 */
static inline double orc_bilin_f(const float *base, long s1, long s2, long n1, long n2,
                                 double q1, double q2, int tex8)
{
    double f1 = floor(q1), f2 = floor(q2);
    long k1 = (long)f1, k2 = (long)f2;
    double a1 = orc_frac_weight(q1 - f1, tex8);
    double a2 = orc_frac_weight(q2 - f2, tex8);
    if (k1 < -1 || k1 >= n1 || k2 < -1 || k2 >= n2) return 0.0;
    double v00 = 0, v10 = 0, v01 = 0, v11 = 0;
    int in1a = (k1 >= 0), in1b = (k1 + 1 < n1);
    int in2a = (k2 >= 0), in2b = (k2 + 1 < n2);
    if (in1a && in2a) v00 = base[k1 * s1 + k2 * s2];
    if (in1b && in2a) v10 = base[(k1 + 1) * s1 + k2 * s2];
    if (in1a && in2b) v01 = base[k1 * s1 + (k2 + 1) * s2];
    if (in1b && in2b) v11 = base[(k1 + 1) * s1 + (k2 + 1) * s2];
    return (1 - a1) * (1 - a2) * v00 + a1 * (1 - a2) * v10 + (1 - a1) * a2 * v01 + a1 * a2 * v11;
}

/* Transpose of orc_bilin_f: scatter w into the (up to) four texels. */
static inline void orc_bilin_scatter(double *base, long s1, long s2, long n1, long n2,
                                     double q1, double q2, double w)
{
    double f1 = floor(q1), f2 = floor(q2);
    long k1 = (long)f1, k2 = (long)f2;
    double a1 = q1 - f1, a2 = q2 - f2;
    if (k1 < -1 || k1 >= n1 || k2 < -1 || k2 >= n2) return;
    int in1a = (k1 >= 0), in1b = (k1 + 1 < n1);
    int in2a = (k2 >= 0), in2b = (k2 + 1 < n2);
    if (in1a && in2a) base[k1 * s1 + k2 * s2] += (1 - a1) * (1 - a2) * w;
    if (in1b && in2a) base[(k1 + 1) * s1 + k2 * s2] += a1 * (1 - a2) * w;
    if (in1a && in2b) base[k1 * s1 + (k2 + 1) * s2] += (1 - a1) * a2 * w;
    if (in1b && in2b) base[(k1 + 1) * s1 + (k2 + 1) * s2] += a1 * a2 * w;
}

/* ------------------------------------------------------------------------- */
/* 3D forward projection: cone (cuda/3d/cone_fp.cu) and par3d                 */
/* (cuda/3d/par3d_fp.cu)                                                      */
/* ------------------------------------------------------------------------- */

enum { ORC_PAR3D = 1, ORC_CONE = 2 };

typedef struct {
    int kind;
    const double *views;
    long nx, ny, nz, na, nu, nv;
    double vs[3];
    double out_scale;
    int rays_per_det;
    int tex8;
    const float *vol;
    double *proj;   /* forward: output [nv][na][nu]; transpose: input */
    double *volT;   /* transpose: output [nz][ny][nx] (one per thread slot) */
    const double *projT_in;
    long a_begin;
} orc_fp3d_ctx;

/*
 * Dominant marching axis of a view, computed exactly as the reference's host
 * code does (double expression, then fabsf on its float value):
 * cone: cuda/3d/cone_fp.cu:375-388; par3d: cuda/3d/par3d_fp.cu:474-487.
 */
int orc_dominant_axis3d(int kind, const double *w, long nu, long nv)
{
    float dX, dY, dZ;
    if (kind == ORC_CONE) {
        dX = fabsf((float)(w[0] - (w[3] + (double)nu * w[6] * 0.5f + (double)nv * w[9] * 0.5f)));
        dY = fabsf((float)(w[1] - (w[4] + (double)nu * w[7] * 0.5f + (double)nv * w[10] * 0.5f)));
        dZ = fabsf((float)(w[2] - (w[5] + (double)nu * w[8] * 0.5f + (double)nv * w[11] * 0.5f)));
    } else {
        dX = fabsf((float)w[0]);
        dY = fabsf((float)w[1]);
        dZ = fabsf((float)w[2]);
    }
    if (dX >= dY && dX >= dZ) return 0;
    if (dY >= dX && dY >= dZ) return 1;
    return 2;
}

/*
 * Ray-sum scale factor sqrt(1 + a1^2*f1 + a2^2*f2) * outScale * vs[dir]:
 * SCALE_CUBE / SCALE_NONCUBE (cone_fp.cu:101-112, par3d_fp.cu:101-112) with the
 * per-direction factors chosen in ConeFP_Array_internal (cone_fp.cu:335-370) and
 * Par3DFP_Array_internal (par3d_fp.cu:436-469).  The par3d Y-direction
 * fScale2 = (fY/fY)^2 = 1 (par3d_fp.cu:460) is kept as the reference has it.
 */
static void orc_scale_factors3d(int kind, int dir, const double vs[3], int force_noncube,
                                double *f1, double *f2, double *mul)
{
    int cube = 1;
    if (fabs((double)((float)vs[0] / (float)vs[1]) - 1.0) > 0.00001) cube = 0;
    if (fabs((double)((float)vs[0] / (float)vs[2]) - 1.0) > 0.00001) cube = 0;
    if (cube && !force_noncube) {
        *f1 = 1.0;
        *f2 = 1.0;
        *mul = vs[0];
        return;
    }
    double s1, s2;
    if (dir == 0) {
        s1 = vs[1] / vs[0];
        s2 = vs[2] / vs[0];
        *mul = vs[0];
    } else if (dir == 1) {
        s1 = vs[0] / vs[1];
        s2 = (kind == ORC_PAR3D) ? 1.0 : vs[2] / vs[1];
        *mul = vs[1];
    } else {
        s1 = vs[0] / vs[2];
        s2 = vs[1] / vs[2];
        *mul = vs[2];
    }
    *f1 = s1 * s1;
    *f2 = s2 * s2;
}

/* Geometry of one slice plane for a marching direction. */
static void orc_plane3d(int dir, long nx, long ny, long nz, long *n0, long *n1, long *n2,
                        long *st0, long *st1, long *st2)
{
    if (dir == 0) {          /* slices along x; q1 -> y, q2 -> z */
        *n0 = nx; *n1 = ny; *n2 = nz;
        *st0 = 1; *st1 = nx; *st2 = nx * ny;
    } else if (dir == 1) {   /* slices along y; q1 -> x, q2 -> z */
        *n0 = ny; *n1 = nx; *n2 = nz;
        *st0 = nx; *st1 = 1; *st2 = nx * ny;
    } else {                 /* slices along z; q1 -> x, q2 -> y */
        *n0 = nz; *n1 = nx; *n2 = ny;
        *st0 = nx * ny; *st1 = 1; *st2 = nx;
    }
}

static inline double orc_c(const double *p, int dir, int which)
{
    /* coordinate permutation of DIR_X / DIR_Y / DIR_Z (cone_fp.cu:60-99) */
    static const int perm[3][3] = {{0, 1, 2}, {1, 0, 2}, {2, 0, 1}};
    return p[perm[dir][which]];
}

/*
 * One ray's line parameters: (x_c1, x_c2) = (a1, a2) * x_c0 + (b1, b2).
 * cone: cone_fp.cu:177-204; par3d: par3d_fp.cu:175-201.
 */
static void orc_ray3d(int kind, const double *w, int dir, double fu, double fv,
                      double *a1, double *a2, double *b1, double *b2)
{
    double D[3];
    for (int k = 0; k < 3; ++k)
        D[k] = w[3 + k] + 0.5 * w[6 + k] + 0.5 * w[9 + k] + fu * w[6 + k] + fv * w[9 + k];
    if (kind == ORC_CONE) {
        const double *S = w;
        double s0 = orc_c(S, dir, 0), s1 = orc_c(S, dir, 1), s2 = orc_c(S, dir, 2);
        double d0 = orc_c(D, dir, 0), d1 = orc_c(D, dir, 1), d2 = orc_c(D, dir, 2);
        *a1 = (s1 - d1) / (s0 - d0);
        *a2 = (s2 - d2) / (s0 - d0);
        *b1 = s1 - *a1 * s0;
        *b2 = s2 - *a2 * s0;
    } else {
        const double *R = w;
        double r0 = orc_c(R, dir, 0), r1 = orc_c(R, dir, 1), r2 = orc_c(R, dir, 2);
        double d0 = orc_c(D, dir, 0), d1 = orc_c(D, dir, 1), d2 = orc_c(D, dir, 2);
        *a1 = r1 / r0;
        *a2 = r2 / r0;
        *b1 = d1 - *a1 * d0;
        *b2 = d2 - *a2 * d0;
    }
}

/* Work items are (view, detector row) pairs so a few views still spread over
 * all threads. */
static void orc_fp3d_range(void *vctx, long begin, long end)
{
    orc_fp3d_ctx *c = (orc_fp3d_ctx *)vctx;
    const long R = c->rays_per_det;
    for (long item = begin; item < end; ++item) {
        long a = c->a_begin + item / c->nv;
        long v = item % c->nv;
        const double *w = c->views + 12 * a;
        int dir = orc_dominant_axis3d(c->kind, w, c->nu, c->nv);
        long n0, n1, n2, st0, st1, st2;
        orc_plane3d(dir, c->nx, c->ny, c->nz, &n0, &n1, &n2, &st0, &st1, &st2);
        double f1, f2, mul;
        orc_scale_factors3d(c->kind, dir, c->vs, R > 1, &f1, &f2, &mul);
        {
            for (long u = 0; u < c->nu; ++u) {
                double acc = 0.0;
                double parsum = 0.0;  /* par3d supersampling scales after the sum */
                double pa1 = 0, pa2 = 0;
                for (long iu = 0; iu < R; ++iu) {
                    for (long iv = 0; iv < R; ++iv) {
                        double fu = (double)u, fv = (double)v;
                        if (R > 1) {
                            fu = u - 0.5 + 0.5 / R + (double)iu / R;
                            fv = v - 0.5 + 0.5 / R + (double)iv / R;
                        }
                        double a1, a2, b1, b2;
                        orc_ray3d(c->kind, w, dir, fu, fv, &a1, &a2, &b1, &b2);
                        double sum = 0.0;
                        for (long s = 0; s < n0; ++s) {
                            double x0 = s - 0.5 * n0 + 0.5;
                            double q1 = a1 * x0 + b1 + 0.5 * n1 - 0.5;
                            double q2 = a2 * x0 + b2 + 0.5 * n2 - 0.5;
                            sum += orc_bilin_f(c->vol + s * st0, st1, st2, n1, n2, q1, q2, c->tex8);
                        }
                        double sc = sqrt(a1 * a1 * f1 + a2 * a2 * f2 + 1.0) * c->out_scale * mul;
                        if (c->kind == ORC_CONE) {
                            acc += sum * sc;
                        } else {
                            parsum += sum;
                            pa1 = a1;
                            pa2 = a2;
                        }
                    }
                }
                if (c->kind == ORC_PAR3D) {
                    double sc = sqrt(pa1 * pa1 * f1 + pa2 * pa2 * f2 + 1.0) * c->out_scale * mul;
                    acc = parsum * sc;
                }
                acc /= (double)(R * R);
                c->proj[(v * c->na + a) * c->nu + u] = acc;
            }
        }
    }
}

/*
 * Forward projection of views [a_begin, a_end).  Writes proj[v][a][u] for those
 * views (other entries untouched).  Reference: ConeFP / Par3DFP
 * (cuda/3d/cone_fp.cu:444-504, cuda/3d/par3d_fp.cu:564-603).
 */
int orc_fp3d(int kind, const double *views, long nx, long ny, long nz, long na, long nu, long nv,
             const double *vs, double out_scale, int rays_per_det, int tex8,
             const float *vol, double *proj, long a_begin, long a_end, int nthreads)
{
    if (kind != ORC_CONE && kind != ORC_PAR3D) return 1;
    if (rays_per_det < 1) return 1;
    orc_fp3d_ctx c;
    memset(&c, 0, sizeof(c));
    c.kind = kind; c.views = views;
    c.nx = nx; c.ny = ny; c.nz = nz; c.na = na; c.nu = nu; c.nv = nv;
    c.vs[0] = vs[0]; c.vs[1] = vs[1]; c.vs[2] = vs[2];
    c.out_scale = out_scale; c.rays_per_det = rays_per_det; c.tex8 = tex8;
    c.vol = vol; c.proj = proj; c.a_begin = a_begin;
    orc_parallel(orc_fp3d_range, &c, (a_end - a_begin) * nv, nthreads);
    return 0;
}

/*
 * Sum of squared linear-interpolation weights of one axis at texture
 * coordinate x (texel centres at i + 0.5, zero border), the piecewise form of
 * dirWeights (cuda/3d/par3d_fp.cu:329-340).
 */
static double orc_dir_sqw(double x, double n)
{
    if (x <= -0.5) return 0.0;
    if (x <= 0.5) return (x + 0.5) * (x + 0.5);
    if (x <= n - 0.5) {
        double t = x + 0.5 - floor(x + 0.5);
        return t * t + (1.0 - t) * (1.0 - t);
    }
    if (x <= n + 0.5) return (n + 0.5 - x) * (n + 0.5 - x);
    return 0.0;
}

/*
 * "sum_square_weights" forward projection of a parallel-beam geometry: per
 * ray, the sum over the dominant axis's slices of the product of both plane
 * axes' squared interpolation weights, times the squared ray-length factor
 * with the non-cube scales (par3D_FP_SumSqW_t, cuda/3d/par3d_fp.cu:343-415;
 * host Par3DFP_SumSqW, par3d_fp.cu:607-703, which always uses SCALE_NONCUBE
 * and the Y-direction fScale2 = (fY/fY)^2).  No volume is read.  Writes
 * proj[v][a][u] (rays_per_det = 1 only, as the reference).
 */
int orc_par3d_sumsqw(const double *views, long nx, long ny, long nz, long na, long nu, long nv,
                     const double *vs, double out_scale, double *proj)
{
    for (long a = 0; a < na; ++a) {
        const double *w = views + 12 * a;
        int dir = orc_dominant_axis3d(ORC_PAR3D, w, nu, nv);
        long n0, n1, n2, st0, st1, st2;
        orc_plane3d(dir, nx, ny, nz, &n0, &n1, &n2, &st0, &st1, &st2);
        double f1, f2, mul;
        orc_scale_factors3d(ORC_PAR3D, dir, vs, 1, &f1, &f2, &mul);
        for (long v = 0; v < nv; ++v) {
            for (long u = 0; u < nu; ++u) {
                double a1, a2, b1, b2;
                orc_ray3d(ORC_PAR3D, w, dir, (double)u, (double)v, &a1, &a2, &b1, &b2);
                double sum = 0.0;
                for (long s = 0; s < n0; ++s) {
                    double x0 = s - 0.5 * n0 + 0.5;
                    /* texture coordinates: index-space position + 0.5 */
                    double t1 = a1 * x0 + b1 + 0.5 * n1;
                    double t2 = a2 * x0 + b2 + 0.5 * n2;
                    sum += orc_dir_sqw(t1, (double)n1) * orc_dir_sqw(t2, (double)n2);
                }
                double sc = sqrt(a1 * a1 * f1 + a2 * a2 * f2 + 1.0) * out_scale * mul;
                proj[(v * na + a) * nu + u] = sum * sc * sc;
            }
        }
    }
    return 0;
}

/*
 * Exact transpose of orc_fp3d (rays_per_det = 1): vol += A^T proj.  Single
 * threaded; used to check the matched (exact-adjoint) backprojector.
 */
int orc_fp3d_transpose(int kind, const double *views, long nx, long ny, long nz, long na, long nu,
                       long nv, const double *vs, double out_scale, const double *proj, double *vol)
{
    if (kind != ORC_CONE && kind != ORC_PAR3D) return 1;
    for (long a = 0; a < na; ++a) {
        const double *w = views + 12 * a;
        int dir = orc_dominant_axis3d(kind, w, nu, nv);
        long n0, n1, n2, st0, st1, st2;
        orc_plane3d(dir, nx, ny, nz, &n0, &n1, &n2, &st0, &st1, &st2);
        double f1, f2, mul;
        orc_scale_factors3d(kind, dir, vs, 0, &f1, &f2, &mul);
        for (long v = 0; v < nv; ++v) {
            for (long u = 0; u < nu; ++u) {
                double a1, a2, b1, b2;
                orc_ray3d(kind, w, dir, (double)u, (double)v, &a1, &a2, &b1, &b2);
                double sc = sqrt(a1 * a1 * f1 + a2 * a2 * f2 + 1.0) * out_scale * mul;
                double val = proj[(v * na + a) * nu + u] * sc;
                if (val == 0.0) continue;
                for (long s = 0; s < n0; ++s) {
                    double x0 = s - 0.5 * n0 + 0.5;
                    double q1 = a1 * x0 + b1 + 0.5 * n1 - 0.5;
                    double q2 = a2 * x0 + b2 + 0.5 * n2 - 0.5;
                    orc_bilin_scatter(vol + s * st0, st1, st2, n1, n2, q1, q2, val);
                }
            }
        }
    }
    return 0;
}

/* ------------------------------------------------------------------------- */
/* 3D backprojection: cone (cuda/3d/cone_bp.cu) and par3d (cuda/3d/par3d_bp.cu) */
/* ------------------------------------------------------------------------- */

enum { ORC_KER_DEFAULT = 0, ORC_KER_FDK = 2, ORC_KER_2D = 3 };

static inline double det3x(const double *b, const double *c) { return b[1] * c[2] - b[2] * c[1]; }
static inline double det3y(const double *b, const double *c) { return -(b[0] * c[2] - b[2] * c[0]); }
static inline double det3z(const double *b, const double *c) { return b[0] * c[1] - b[1] * c[0]; }
static inline double det3(const double *a, const double *b, const double *c)
{
    return a[0] * det3x(b, c) + a[1] * det3y(b, c) + a[2] * det3z(b, c);
}
static inline double scaled_cross_norm(const double *a, const double *b, const double *sc)
{
    double x = det3x(a, b) * sc[1] * sc[2];
    double y = det3y(a, b) * sc[0] * sc[2];
    double z = det3z(a, b) * sc[0] * sc[1];
    return sqrt(x * x + y * y + z * z);
}

/* Per-view BP coefficients: texture u = (Nu.w + Nu.xyz.x) / Den, v likewise. */
typedef struct {
    double nu[4], nv[4], den[4];  /* .w stored at index 3 */
    double par_scale;             /* par3d: weight per view */
} orc_bpview;

/*
 * Cone: transferConstants (cone_bp.cu:221-302); par3d: transferConstants
 * (par3d_bp.cu:202-244).  Computed in double exactly as there; the model is
 * then evaluated in double instead of float.
 */
static void orc_bp_coeffs(int kind, int kernel, const double *w, const double *vs, orc_bpview *o)
{
    const double *u = w + 6, *v = w + 9, *d = w + 3;
    if (kind == ORC_CONE) {
        const double *s = w;
        double smd[3] = {s[0] - d[0], s[1] - d[1], s[2] - d[2]};
        double scale;
        if (kernel == ORC_KER_FDK) {
            scale = 1.0 / det3(u, v, s);
        } else if (kernel == ORC_KER_2D) {
            double ez[3] = {0, 0, 1};
            scale = scaled_cross_norm(u, ez, vs) / det3(u, v, smd);
        } else {
            scale = sqrt(scaled_cross_norm(u, v, vs)) / det3(u, v, smd);
        }
        o->nu[3] = scale * det3(s, v, d);
        o->nu[0] = scale * det3x(v, smd);
        o->nu[1] = scale * det3y(v, smd);
        o->nu[2] = scale * det3z(v, smd);
        o->nv[3] = -scale * det3(s, u, d);
        o->nv[0] = -scale * det3x(u, smd);
        o->nv[1] = -scale * det3y(u, smd);
        o->nv[2] = -scale * det3z(u, smd);
        o->den[3] = (kernel == ORC_KER_FDK) ? 1.0 : scale * det3(u, v, s);
        o->den[0] = -scale * det3x(u, v);
        o->den[1] = -scale * det3y(u, v);
        o->den[2] = -scale * det3z(u, v);
        o->par_scale = 0.0;
    } else {
        const double *r = w;
        double den = det3(r, u, v);
        o->nu[0] = -det3x(r, v) / den;
        o->nu[1] = -det3y(r, v) / den;
        o->nu[2] = -det3z(r, v) / den;
        o->nu[3] = -det3(r, d, v) / den;
        o->nv[0] = det3x(r, u) / den;
        o->nv[1] = det3y(r, u) / den;
        o->nv[2] = det3z(r, u) / den;
        o->nv[3] = det3(r, d, u) / den;
        if (kernel == ORC_KER_2D) {
            double ez[3] = {0, 0, 1};
            o->par_scale = 1.0 / scaled_cross_norm(u, ez, vs);
        } else {
            o->par_scale = 1.0 / scaled_cross_norm(u, v, vs);
        }
    }
}

typedef struct {
    int kind, kernel, tex8;
    const double *views;
    long nx, ny, nz, na, nu, nv;
    double vs[3];
    double out_scale;
    int rays_per_voxel;
    const float *proj;
    double *vol;
    orc_bpview *co;
} orc_bp3d_ctx;

static inline double orc_bp_sample(const orc_bp3d_ctx *c, long a, double x, double y, double z)
{
    const orc_bpview *o = &c->co[a];
    double U = o->nu[3] + x * o->nu[0] + y * o->nu[1] + z * o->nu[2];
    double V = o->nv[3] + x * o->nv[0] + y * o->nv[1] + z * o->nv[2];
    double wgt;
    if (c->kind == ORC_CONE) {
        double den = o->den[3] + x * o->den[0] + y * o->den[1] + z * o->den[2];
        double fr = 1.0 / den;
        U *= fr;
        V *= fr;
        wgt = (c->kernel == ORC_KER_2D) ? fr : fr * fr;
    } else {
        wgt = o->par_scale;
    }
    /* texture coordinates (U, angle + 0.5, V); texel centres at +0.5 */
    const float *plane = c->proj + a * c->nu;
    double val = orc_bilin_f(plane, 1, c->na * c->nu, c->nu, c->nv, U - 0.5, V - 0.5, c->tex8);
    return val * wgt;
}

static void orc_bp3d_range(void *vctx, long begin, long end)
{
    orc_bp3d_ctx *c = (orc_bp3d_ctx *)vctx;
    const long R = c->rays_per_voxel;
    double outs;
    if (c->kind == ORC_CONE && c->kernel == ORC_KER_FDK)
        outs = c->out_scale / c->vs[0];   /* cone_bp.cu:323-325 */
    else
        outs = c->out_scale * c->vs[0] * c->vs[1] * c->vs[2];
    outs /= (double)(R * R * R);
    /* [begin, end) are volume rows Z * ny + Y */
    for (long row = begin; row < end; ++row) {
        const long Z = row / c->ny;
        {
            const long Y = row % c->ny;
            for (long X = 0; X < c->nx; ++X) {
                double x = X - 0.5 * c->nx + 0.5;
                double y = Y - 0.5 * c->ny + 0.5;
                double z = Z - 0.5 * c->nz + 0.5;
                double acc = 0.0;
                for (long a = 0; a < c->na; ++a) {
                    if (R == 1) {
                        acc += orc_bp_sample(c, a, x, y, z);
                    } else {
                        for (long i = 0; i < R; ++i)
                            for (long j = 0; j < R; ++j)
                                for (long k = 0; k < R; ++k)
                                    acc += orc_bp_sample(c, a, x - 0.5 + 0.5 / R + (double)i / R,
                                                         y - 0.5 + 0.5 / R + (double)j / R,
                                                         z - 0.5 + 0.5 / R + (double)k / R);
                    }
                }
                c->vol[(Z * c->ny + Y) * c->nx + X] = acc * outs;
            }
        }
    }
}

/*
 * Backprojection of all views into slices [z_begin, z_end) of vol[z][y][x]
 * (written, not accumulated).  kernel: 0 default, 2 fdk_weighting, 3
 * 2d_weighting.  Reference: ConeBP (cuda/3d/cone_bp.cu:55-217,305-401),
 * Par3DBP (cuda/3d/par3d_bp.cu:55-198,246-335).
 */
int orc_bp3d(int kind, int kernel, const double *views, long nx, long ny, long nz, long na, long nu,
             long nv, const double *vs, double out_scale, int rays_per_voxel, int tex8,
             const float *proj, double *vol, long z_begin, long z_end, int nthreads)
{
    if (kind != ORC_CONE && kind != ORC_PAR3D) return 1;
    if (kind == ORC_PAR3D && kernel == ORC_KER_FDK) return 1;
    if (rays_per_voxel < 1) return 1;
    orc_bp3d_ctx c;
    memset(&c, 0, sizeof(c));
    c.kind = kind; c.kernel = kernel; c.tex8 = tex8; c.views = views;
    c.nx = nx; c.ny = ny; c.nz = nz; c.na = na; c.nu = nu; c.nv = nv;
    c.vs[0] = vs[0]; c.vs[1] = vs[1]; c.vs[2] = vs[2];
    c.out_scale = out_scale; c.rays_per_voxel = rays_per_voxel;
    c.proj = proj; c.vol = vol;
    c.co = (orc_bpview *)malloc(sizeof(orc_bpview) * (size_t)na);
    if (!c.co) return 2;
    for (long a = 0; a < na; ++a) orc_bp_coeffs(kind, kernel, views + 12 * a, vs, &c.co[a]);
    /* rows Z * ny + Y of slices [z_begin, z_end) are split across threads */
    long n = (z_end - z_begin) * ny;
    if (nthreads <= 1 || n <= 1) {
        orc_bp3d_range(&c, z_begin * ny, z_end * ny);
    } else {
        if (nthreads > 256) nthreads = 256;
        if (nthreads > n) nthreads = (int)n;
        pthread_t th[256];
        orc_job jobs[256];
        for (int t = 0; t < nthreads; ++t) {
            jobs[t].fn = orc_bp3d_range;
            jobs[t].ctx = &c;
            jobs[t].begin = z_begin * ny + n * t / nthreads;
            jobs[t].end = z_begin * ny + n * (t + 1) / nthreads;
            pthread_create(&th[t], NULL, orc_thread_main, &jobs[t]);
        }
        for (int t = 0; t < nthreads; ++t) pthread_join(th[t], NULL);
    }
    free(c.co);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* FDK weighting (cuda/3d/fdk.cu:70-163, 168-264, 415-472)                    */
/* ------------------------------------------------------------------------- */

/*
 * Circular parameters recovered from view 0 and the per-view angles, exactly as
 * FDK() does on the host (fdk.cu:425-445).  out[0..4] = fSrcOrigin, fDetOrigin,
 * fDetUSize, fDetVSize, fZShift (as floats), angles[na] = -atan2(sx, sy) + pi.
 */
void orc_fdk_params(const double *views, long na, long nu, long nv, float *out, float *angles)
{
    const double *p0 = views;
    float fDetCX = (float)(p0[3] + 0.5 * nu * p0[6]);
    float fDetCY = (float)(p0[4] + 0.5 * nu * p0[7]);
    float fDetCZ = (float)(p0[5] + 0.5 * nv * p0[11]);
    out[0] = (float)sqrt(p0[0] * p0[0] + p0[1] * p0[1]);
    out[1] = sqrtf(fDetCX * fDetCX + fDetCY * fDetCY);  /* float sqrt, as fdk.cu:434 */
    out[2] = (float)sqrt(p0[6] * p0[6] + p0[7] * p0[7]);
    out[3] = (float)fabs(p0[11]);
    out[4] = (float)(fDetCZ - p0[2]);
    for (long i = 0; i < na; ++i)
        angles[i] = (float)(-atan2(views[12 * i + 0], views[12 * i + 1]) + M_PI);
}

/*
 * FDK cosine/magnification pre-weight, in place on proj[v][a][u]
 * (devFDK_preweight, fdk.cu:70-113), evaluated in double.
 */
void orc_fdk_preweight(double *proj, long na, long nu, long nv, double src_origin, double det_origin,
                       double zshift, double det_usize, double det_vsize)
{
    double L = src_origin + det_origin;
    double W2 = L / (det_usize * src_origin);
    double W = L * W2 * (M_PI / 2.0) / (double)na;
    for (long v = 0; v < nv; ++v) {
        double fv = (v - 0.5 * nv + 0.5) * det_vsize + zshift;
        for (long a = 0; a < na; ++a) {
            for (long u = 0; u < nu; ++u) {
                double fu = (u - 0.5 * nu + 0.5) * det_usize;
                double rl = sqrt(L * L + fu * fu + fv * fv);
                proj[(v * na + a) * nu + u] *= W / rl;
            }
        }
    }
}

/*
 * Parker short-scan weight (devFDK_ParkerWeight, fdk.cu:115-163) with the
 * angle range logic of FDK_PreWeight (fdk.cu:195-251).  rel_angles and scale
 * are computed by the caller (orc_parker_setup) in float as the reference does.
 */
void orc_parker_setup(const float *angles, long na, long nu, double src_origin, double det_origin,
                      double det_usize, float *rel, float *scale, float *central_fan)
{
    float fdA = angles[1] - angles[0];
    while (fdA < -M_PI) fdA += 2 * M_PI;
    while (fdA >= M_PI) fdA -= 2 * M_PI;
    float base = (fdA >= 0.0f) ? angles[0] : angles[na - 1];
    for (long i = 0; i < na; ++i) {
        float f = angles[i] - base;
        while (f >= 2 * M_PI) f -= 2 * M_PI;
        while (f < 0) f += 2 * M_PI;
        rel[i] = f;
    }
    float range = fabsf(rel[na - 1] - rel[0]);
    range /= (float)(na - 1);
    range *= (float)na;
    *scale = (float)(range / M_PI);
    *central_fan = fabsf(atanf((float)det_usize * (nu * 0.5f) / (float)(src_origin + det_origin)));
}

void orc_parker_weight(double *proj, long na, long nu, long nv, double src_origin, double det_origin,
                       double det_usize, const float *rel, double scale, double central_fan)
{
    double L = src_origin + det_origin;
    for (long a = 0; a < na; ++a) {
        double beta = rel[a];
        for (long u = 0; u < nu; ++u) {
            double fu = (u - 0.5 * nu + 0.5) * det_usize;
            double g = atan(fu / L);
            double wgt;
            if (beta <= 0.0) wgt = 0.0;
            else if (beta <= 2.0 * (central_fan + g)) {
                wgt = sin((M_PI / 4.0) * beta / (central_fan + g));
                wgt *= wgt;
            } else if (beta <= M_PI + 2 * g) wgt = 1.0;
            else if (beta <= M_PI + 2 * central_fan) {
                wgt = sin((M_PI / 4.0) * (M_PI + 2.0 * central_fan - beta) / (central_fan - g));
                wgt *= wgt;
            } else wgt = 0.0;
            wgt *= scale;
            for (long v = 0; v < nv; ++v) proj[(v * na + a) * nu + u] *= wgt;
        }
    }
}

/*
 * Ram-Lak ramp filter along u, as the exact Toeplitz product it equals:
 * y[i] = sum_j 2 h(|i-j|) x[j], h(0) = 1/4, h(odd k) = -1/(pi k)^2, h(even) = 0.
 * Reference: generateRampFilter (src/Filters.cpp:41-69), genFilter
 * (src/Filters.cpp:133-152), FDK_Filter (cuda/3d/fdk.cu:266-412); the zero
 * padding to nextpow2(2*nu) >= 2*nu keeps the circular FFT convolution free of
 * wrap-around, so it is identically this Toeplitz product.
 */
typedef struct { double *rows; long nrows, n; const double *taps; } orc_ramp_ctx;

static void orc_ramp_range(void *vctx, long begin, long end)
{
    orc_ramp_ctx *c = (orc_ramp_ctx *)vctx;
    double *tmp = (double *)malloc(sizeof(double) * (size_t)c->n);
    for (long r = begin; r < end; ++r) {
        double *x = c->rows + r * c->n;
        for (long i = 0; i < c->n; ++i) {
            double acc = 0.0;
            for (long j = 0; j < c->n; ++j) acc += c->taps[labs(i - j)] * x[j];
            tmp[i] = acc;
        }
        memcpy(x, tmp, sizeof(double) * (size_t)c->n);
    }
    free(tmp);
}

void orc_ramp_taps(long n, double *taps)
{
    for (long k = 0; k < n; ++k) {
        if (k == 0) taps[k] = 2.0 * 0.25;
        else if (k & 1) taps[k] = 2.0 * (-1.0 / ((M_PI * k) * (M_PI * k)));
        else taps[k] = 0.0;
    }
}

void orc_ramp_filter_rows(double *rows, long nrows, long n, int nthreads)
{
    double *taps = (double *)malloc(sizeof(double) * (size_t)n);
    orc_ramp_taps(n, taps);
    orc_ramp_ctx c = {rows, nrows, n, taps};
    orc_parallel(orc_ramp_range, &c, nrows, nthreads);
    free(taps);
}

/*
 * Any row filter as its exact Toeplitz product (the reference's zero-padded
 * FFT convolution, cuda/3d/fdk.cu:292-398 and cuda/2d/fft.cu:52-110, with the
 * row at offset 0 of nextpow2(2n) samples, equals the linear convolution with
 * the inverse transform g of the filter spectrum):
 *   y[i] = sum_j g[i - j] x[j],  g of offset d at taps[set * (2n - 1) + d + n - 1].
 * Row r uses set (r % set_mod) when nsets > 1 (one filter per view), else set 0.
 */
typedef struct { double *rows; long nrows, n; const double *taps; long nsets, set_mod; } orc_toep_ctx;

static void orc_toep_range(void *vctx, long begin, long end)
{
    orc_toep_ctx *c = (orc_toep_ctx *)vctx;
    const long n = c->n;
    double *tmp = (double *)malloc(sizeof(double) * (size_t)n);
    for (long r = begin; r < end; ++r) {
        double *x = c->rows + r * n;
        const long set = c->nsets > 1 ? r % c->set_mod : 0;
        const double *g = c->taps + set * (2 * n - 1) + (n - 1);
        for (long i = 0; i < n; ++i) {
            double acc = 0.0;
            for (long j = 0; j < n; ++j) acc += g[i - j] * x[j];
            tmp[i] = acc;
        }
        memcpy(x, tmp, sizeof(double) * (size_t)n);
    }
    free(tmp);
}

void orc_toeplitz_rows(double *rows, long nrows, long n, const double *taps, long nsets, long set_mod, int nthreads)
{
    orc_toep_ctx c = {rows, nrows, n, taps, nsets, set_mod > 0 ? set_mod : 1};
    orc_parallel(orc_toep_range, &c, nrows, nthreads);
}

/* ------------------------------------------------------------------------- */
/* 2D parallel FP (cuda/2d/par_fp.cu) and BP (cuda/2d/par_bp.cu)              */
/* ------------------------------------------------------------------------- */

/*
 * getParParameters (src/GeometryUtil2D.cpp:107-131): angle, detector size and
 * offset of a parallel view, as floats.
 */
void orc_par_parameters(const float *p, long ndets, float *angle, float *detsize, float *offset)
{
    double ux = p[4], uy = p[5];
    double t = (ux * p[0] + uy * p[1]) / ((double)p[0] * p[0] + (double)p[1] * p[1]);
    ux -= t * p[0];
    uy -= t * p[1];
    *angle = (float)atan2(uy, ux);
    double norm2 = uy * uy + ux * ux;
    *detsize = (float)sqrt(norm2);
    *offset = (float)(-0.5 * ndets - (p[3] * uy + p[2] * ux) / norm2);
}

/*
 * 2D parallel FP over all views (FPhorizontal_simple / FPvertical_simple,
 * par_fp.cu:53-200, orientation choice par_fp.cu:271-272), supersampling
 * rays_per_det.  vol[row][col] (W cols, H rows), sino[a][det] written.
 */
void orc_par_fp(const float *views, long na, long ndet, long W, long H, double out_scale,
                int rays_per_det, int tex8, const float *vol, double *sino)
{
    for (long a = 0; a < na; ++a) {
        const float *p = views + 6 * a;
        float th, ds, off;
        orc_par_parameters(p, ndet, &th, &ds, &off);
        double c = cos((double)th), s = sin((double)th);
        int vertical = fabsf(p[0]) <= fabsf(p[1]);
        for (long d = 0; d < ndet; ++d) {
            double acc = 0.0;
            double detstep, slicestep, corr, p0;
            long nslices;
            if (!vertical) {
                detstep = -ds / s;
                slicestep = c / s;
                corr = out_scale / fabs(s);
                nslices = W;
                p0 = (d - 0.5 * ndet + 0.5 - off) * detstep + (0 - 0.5 * W + 0.5) * slicestep + 0.5 * H;
            } else {
                detstep = ds / c;
                slicestep = s / c;
                corr = out_scale / fabs(c);
                nslices = H;
                p0 = (d - 0.5 * ndet + 0.5 - off) * detstep + (0 - 0.5 * H + 0.5) * slicestep + 0.5 * W;
            }
            long R = rays_per_det;
            for (long r = 0; r < R; ++r) {
                double pr = p0 + ((-0.5 * R + 0.5) / R + (double)r / R) * detstep;
                for (long sl = 0; sl < nslices; ++sl) {
                    double P = pr + sl * slicestep;  /* texture coordinate */
                    if (!vertical)  /* tex2D(x = slice + 0.5, y = P): column sl, row P - 0.5 */
                        acc += orc_bilin_f(vol + sl, W, 1, H, 1, P - 0.5, 0.0, tex8);
                    else            /* tex2D(x = P, y = slice + 0.5): row sl, column P - 0.5 */
                        acc += orc_bilin_f(vol + sl * W, 1, 1, W, 1, P - 0.5, 0.0, tex8);
                }
            }
            sino[a * ndet + d] = acc * corr / (double)R;
        }
    }
}

/* 2D parallel BP (devBP / devBP_SS, par_bp.cu:52-137; constants par_bp.cu:163-191). */
void orc_par_bp(const float *views, long na, long ndet, long W, long H, double out_scale,
                int rays_per_pixel, int tex8, const float *sino, double *vol)
{
    double *sc = (double *)malloc(sizeof(double) * 4 * (size_t)na);
    for (long a = 0; a < na; ++a) {
        const float *p = views + 6 * a;
        double d = (double)p[4] * p[1] - (double)p[5] * p[0];
        sc[4 * a + 0] = p[1] / d;                                   /* scaled cos */
        sc[4 * a + 1] = -p[0] / d;                                  /* scaled sin */
        sc[4 * a + 2] = ((double)p[3] * p[0] - (double)p[2] * p[1]) / d;  /* offset */
        sc[4 * a + 3] = sqrt((double)p[0] * p[0] + (double)p[1] * p[1]) / fabs(d);
    }
    long R = rays_per_pixel;
    for (long Y = 0; Y < H; ++Y) {
        for (long X = 0; X < W; ++X) {
            double acc = 0.0;
            for (long a = 0; a < na; ++a) {
                for (long i = 0; i < R; ++i) {
                    for (long j = 0; j < R; ++j) {
                        double x = X - 0.5 * W + 0.5, y = Y - 0.5 * H + 0.5;
                        if (R > 1) {
                            x += -0.5 + 0.5 / R + (double)i / R;
                            y += -0.5 + 0.5 / R + (double)j / R;
                        }
                        double T = x * sc[4 * a] - y * sc[4 * a + 1] + sc[4 * a + 2];
                        acc += orc_bilin_f(sino + a * ndet, 1, 1, ndet, 1, T - 0.5, 0.0, tex8) * sc[4 * a + 3];
                    }
                }
            }
            vol[Y * W + X] = acc * out_scale / (double)(R * R);
        }
    }
    free(sc);
}

/* ------------------------------------------------------------------------- */
/* 2D fan FP (cuda/2d/fan_fp.cu) and BP (cuda/2d/fan_bp.cu)                   */
/* ------------------------------------------------------------------------- */

/* 2D fan FP (FanFPhorizontal / FanFPvertical, fan_fp.cu:55-193). */
void orc_fan_fp(const float *views, long na, long ndet, long W, long H, double out_scale,
                int rays_per_det, int tex8, const float *vol, double *sino)
{
    long R = rays_per_det;
    for (long a = 0; a < na; ++a) {
        const float *p = views + 6 * a;
        double sx = p[0], sy = p[1], dsx = p[2], dsy = p[3], ux = p[4], uy = p[5];
        for (long d = 0; d < ndet; ++d) {
            /* per-ray orientation, float arithmetic with contraction as nvcc emits it */
            float fdx = fabsf(fmaf((float)d, p[4], p[2]) + 0.5f - p[0]);
            float fdy = fabsf(fmaf((float)d, p[5], p[3]) + 0.5f - p[1]);
            int horizontal = !(fdy > fdx);
            double acc = 0.0;
            for (long r = 0; r < R; ++r) {
                double fdet = d + (0.5 + r) / R;
                double DX = dsx + fdet * ux, DY = dsy + fdet * uy;
                double sum = 0.0, corr;
                if (horizontal) {
                    double alpha = (sy - DY) / (sx - DX);
                    double beta = sy - alpha * sx;
                    corr = sqrt(alpha * alpha + 1.0) * out_scale / R;
                    for (long sl = 0; sl < W; ++sl) {
                        double fy = -alpha * (sl - 0.5 * W + 0.5) - beta + 0.5 * H;  /* row + 0.5 */
                        sum += orc_bilin_f(vol + sl, W, 1, H, 1, fy - 0.5, 0.0, tex8);
                    }
                } else {
                    double alpha = (sx - DX) / (sy - DY);
                    double beta = sx - alpha * sy;
                    corr = sqrt(alpha * alpha + 1.0) * out_scale / R;
                    for (long sl = 0; sl < H; ++sl) {
                        double fx = -alpha * (sl - 0.5 * H + 0.5) + beta + 0.5 * W;  /* col + 0.5 */
                        sum += orc_bilin_f(vol + sl * W, 1, 1, W, 1, fx - 0.5, 0.0, tex8);
                    }
                }
                acc += sum * corr;
            }
            sino[a * ndet + d] = acc;
        }
    }
}

/*
 * 2D fan BP (devFanBP<FBPWEIGHT> / devFanBP_SS, fan_bp.cu:57-161; constants
 * fan_bp.cu:225-279).  fbp != 0 selects the FBP weighting 1/Den^2.
 */
void orc_fan_bp(const float *views, long na, long ndet, long W, long H, double out_scale,
                int rays_per_pixel, int fbp, int tex8, const float *sino, double *vol)
{
    double *cf = (double *)malloc(sizeof(double) * 6 * (size_t)na);
    for (long a = 0; a < na; ++a) {
        const float *p = views + 6 * a;
        double ux = p[4], uy = p[5], sx = p[0], sy = p[1], dx = p[2], dy = p[3];
        double smdx = sx - dx, smdy = sy - dy;
        double scale;
        if (!fbp) scale = sqrt(ux * ux + uy * uy) / (ux * smdy - uy * smdx);
        else scale = 1.0 / (ux * sy - uy * sx);
        cf[6 * a + 0] = scale * (sx * dy - sy * dx);  /* NumC = det2(s, d) */
        cf[6 * a + 1] = scale * smdy;                 /* NumX */
        cf[6 * a + 2] = -scale * smdx;                /* NumY */
        cf[6 * a + 3] = fbp ? 1.0 : scale * (ux * sy - uy * sx);  /* DenC */
        cf[6 * a + 4] = scale * uy;                   /* DenX */
        cf[6 * a + 5] = -scale * ux;                  /* DenY */
    }
    long R = rays_per_pixel;
    for (long Y = 0; Y < H; ++Y) {
        for (long X = 0; X < W; ++X) {
            double acc = 0.0;
            for (long a = 0; a < na; ++a) {
                const double *c = cf + 6 * a;
                for (long i = 0; i < R; ++i) {
                    for (long j = 0; j < R; ++j) {
                        double x = X - 0.5 * W + 0.5;
                        double y = -(Y - 0.5 * H + 0.5);
                        if (R > 1) {
                            x = X - 0.5 * W + 0.5 - 0.5 + 0.5 / R + (double)i / R;
                            y = -(Y - 0.5 * H + 0.5 - 0.5 + 0.5 / R) - (double)j / R;
                        }
                        double num = c[0] + c[1] * x + c[2] * y;
                        double den = c[3] + c[4] * x + c[5] * y;
                        double fr = 1.0 / den;
                        double T = num * fr;
                        double wgt = fbp ? fr * fr : fr;
                        acc += orc_bilin_f(sino + a * ndet, 1, 1, ndet, 1, T - 0.5, 0.0, tex8) * wgt;
                    }
                }
            }
            vol[Y * W + X] = acc * out_scale / (double)(R * R);
        }
    }
    free(cf);
}

/* Version tag so the loader can check it picked up this build. */
/* ------------------------------------------------------------------------- */
/* cone beam on a cylindrical detector (cyl_cone_vec)                         */
/* ------------------------------------------------------------------------- */

/* view w: src[3], det_c[3], det_u[3], det_v[3], radius (SCylConeProjection) */
static void orc_cross(const double *a, const double *b, double *o)
{
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}
static double orc_norm3(const double *a) { return sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]); }

/* getCylConeAxes (src/GeometryUtil3D.cpp:542-561): radial a, tangential b,
 * cylinder centre c. */
static void orc_cyl_axes(const double *w, double *a, double *b, double *c)
{
    const double *s = w, *d = w + 3, *u = w + 6, *v = w + 9;
    double R = w[12], uv[3];
    orc_cross(u, v, uv);
    double k = -R / (orc_norm3(u) * orc_norm3(v));
    for (int i = 0; i < 3; ++i) a[i] = uv[i] * k;
    double m[3], p[3];
    for (int i = 0; i < 3; ++i) {
        m[i] = d[i] - a[i] - s[i];
        p[i] = d[i] + a[i] - s[i];
    }
    if (orc_norm3(m) > orc_norm3(p))
        for (int i = 0; i < 3; ++i) a[i] = -a[i];
    for (int i = 0; i < 3; ++i) {
        c[i] = d[i] - a[i];
        b[i] = u[i] * (R / orc_norm3(u));
    }
}

/* dominant axis of source - detector centre, compared in float
 * (ConeCylFP_Array_internal, cuda/3d/cone_cyl.cu:491-503) */
static int orc_cyl_dir(const double *w)
{
    float dX = fabsf((float)(w[0] - w[3]));
    float dY = fabsf((float)(w[1] - w[4]));
    float dZ = fabsf((float)(w[2] - w[5]));
    if (dX >= dY && dX >= dZ) return 0;
    if (dY >= dX && dY >= dZ) return 1;
    return 2;
}

/*
 * One cylinder ray (cylcone_FP_t, cone_cyl.cu:197-306): slopes a1, a2 in
 * texel steps per slice, offsets b1, b2 (texel units at the marching
 * axis's world origin) and the ray length per slice.  Views are in world
 * units, centred on the volume (convertAstraGeometry_unscaled).
 */
static void orc_cyl_ray(const double *w, int dir, long nu, long nv, long u, long v, const double *vs,
                        double *a1, double *a2, double *b1, double *b2, double *corr)
{
    double A[3], B[3], C[3];
    orc_cyl_axes(w, A, B, C);
    double ut = orc_norm3(w + 6) / w[12];
    double th = (2.0 * u - nu + 1) * 0.5 * ut;
    double dv = v - 0.5 * nv + 0.5;
    double D[3];
    for (int k = 0; k < 3; ++k) D[k] = C[k] + A[k] * cos(th) + B[k] * sin(th) + w[9 + k] * dv;
    double S0 = orc_c(w, dir, 0), S1 = orc_c(w, dir, 1), S2 = orc_c(w, dir, 2);
    double D0 = orc_c(D, dir, 0), D1 = orc_c(D, dir, 1), D2 = orc_c(D, dir, 2);
    double v0 = orc_c(vs, dir, 0), v1 = orc_c(vs, dir, 1), v2 = orc_c(vs, dir, 2);
    double s1 = (S1 - D1) / (S0 - D0), s2 = (S2 - D2) / (S0 - D0);
    *corr = sqrt(s1 * s1 + s2 * s2 + 1.0) * v0;
    *a1 = s1 / v1 * v0;
    *a2 = s2 / v2 * v0;
    *b1 = S1 / v1 - s1 / v1 * S0;
    *b2 = S2 / v2 - s2 / v2 * S0;
}

/*
 * FP (ConeCylFP, cone_cyl.cu:622-682): per ray the bilinear samples (zero
 * border) at every slice s of the dominant axis, texture coordinates
 * a (s + 1/2 - n0/2) + b + n/2, times the ray length per slice and out_scale.
 * views: (na, 13).  proj[v][a][u] written.
 */
int orc_cylcone_fp(const double *views, long nx, long ny, long nz, long na, long nu, long nv, const double *vs,
                   double out_scale, int tex8, const float *vol, double *proj)
{
    for (long a = 0; a < na; ++a) {
        const double *w = views + 13 * a;
        int dir = orc_cyl_dir(w);
        long n0, n1, n2, st0, st1, st2;
        orc_plane3d(dir, nx, ny, nz, &n0, &n1, &n2, &st0, &st1, &st2);
        for (long v = 0; v < nv; ++v) {
            for (long u = 0; u < nu; ++u) {
                double a1, a2, b1, b2, corr;
                orc_cyl_ray(w, dir, nu, nv, u, v, vs, &a1, &a2, &b1, &b2, &corr);
                double sum = 0.0;
                for (long s = 0; s < n0; ++s) {
                    double x0 = s + 0.5 - 0.5 * n0;
                    double q1 = a1 * x0 + b1 + 0.5 * n1 - 0.5;
                    double q2 = a2 * x0 + b2 + 0.5 * n2 - 0.5;
                    sum += orc_bilin_f(vol + s * st0, st1, st2, n1, n2, q1, q2, tex8);
                }
                proj[(v * na + a) * nu + u] = sum * corr * out_scale;
            }
        }
    }
    return 0;
}

/* Exact transpose of orc_cylcone_fp: vol += A^T proj (the model of
 * ConeCylBP_matched, cone_cyl.cu:308-475, 684-749, with out_scale). */
int orc_cylcone_fp_transpose(const double *views, long nx, long ny, long nz, long na, long nu, long nv,
                             const double *vs, double out_scale, const double *proj, double *vol)
{
    for (long a = 0; a < na; ++a) {
        const double *w = views + 13 * a;
        int dir = orc_cyl_dir(w);
        long n0, n1, n2, st0, st1, st2;
        orc_plane3d(dir, nx, ny, nz, &n0, &n1, &n2, &st0, &st1, &st2);
        for (long v = 0; v < nv; ++v) {
            for (long u = 0; u < nu; ++u) {
                double a1, a2, b1, b2, corr;
                orc_cyl_ray(w, dir, nu, nv, u, v, vs, &a1, &a2, &b1, &b2, &corr);
                double val = proj[(v * na + a) * nu + u] * corr * out_scale;
                for (long s = 0; s < n0; ++s) {
                    double x0 = s + 0.5 - 0.5 * n0;
                    double q1 = a1 * x0 + b1 + 0.5 * n1 - 0.5;
                    double q2 = a2 * x0 + b2 + 0.5 * n2 - 0.5;
                    orc_bilin_scatter(vol + s * st0, st1, st2, n1, n2, q1, q2, val);
                }
            }
        }
    }
    return 0;
}

/*
 * Voxel-driven BP (ConeCylBP: dev_cylcone_BP cone_cyl_bp.cu:61-160,
 * constants :162-233, host :235-320): for voxel centre x and view, the ray
 * s + t (x - s) / sqrt|u x v| meets the cylinder (larger root t); the
 * detector is sampled bilinearly (zero border) at angular coordinate
 * asin(b / R) / (|u| / R) + nu/2 and axial coordinate v / |v| + nv/2 of that
 * point; weight t^2; times out_scale and the voxel volume.  vol[z][y][x].
 */
int orc_cylcone_bp(const double *views, long nx, long ny, long nz, long na, long nu, long nv, const double *vs,
                   double out_scale, int tex8, const float *proj, double *vol)
{
    double scale = out_scale * vs[0] * vs[1] * vs[2];
    for (long z = 0; z < nz; ++z)
        for (long y = 0; y < ny; ++y)
            for (long x = 0; x < nx; ++x) vol[(z * ny + y) * nx + x] = 0.0;
    for (long a = 0; a < na; ++a) {
        const double *w = views + 13 * a;
        double A[3], B[3], C[3], uv[3];
        orc_cyl_axes(w, A, B, C);
        double R = w[12], nA = orc_norm3(A), nB = orc_norm3(B), nV = orc_norm3(w + 9);
        orc_cross(w + 6, w + 9, uv);
        double f = sqrt(orc_norm3(uv));
        double an[3], bn[3], vn[3], smc[3];
        for (int k = 0; k < 3; ++k) {
            an[k] = A[k] / nA;
            bn[k] = B[k] / nB;
            vn[k] = w[9 + k] / nV;
            smc[k] = w[k] - C[k];
        }
        double sa = smc[0] * an[0] + smc[1] * an[1] + smc[2] * an[2];
        double sb = smc[0] * bn[0] + smc[1] * bn[1] + smc[2] * bn[2];
        double sc = smc[0] * vn[0] + smc[1] * vn[1] + smc[2] * vn[2];
        double ut = orc_norm3(w + 6) / R;
        for (long z = 0; z < nz; ++z) {
            for (long y = 0; y < ny; ++y) {
                for (long x = 0; x < nx; ++x) {
                    double p[3] = {vs[0] * (x - 0.5 * nx + 0.5), vs[1] * (y - 0.5 * ny + 0.5),
                                   vs[2] * (z - 0.5 * nz + 0.5)};
                    double r[3] = {p[0] - w[0], p[1] - w[1], p[2] - w[2]};
                    double ra = f * (r[0] * an[0] + r[1] * an[1] + r[2] * an[2]);
                    double rb = f * (r[0] * bn[0] + r[1] * bn[1] + r[2] * bn[2]);
                    double rc = f * (r[0] * vn[0] + r[1] * vn[1] + r[2] * vn[2]);
                    double qa = ra * ra + rb * rb, qb = ra * sa + rb * sb, qc = sa * sa + sb * sb - R * R;
                    double disc = qb * qb - qa * qc;
                    if (disc < 0 || qa <= 0) continue;
                    double t = (-qb + sqrt(disc)) / qa;
                    double th = asin((t * rb + sb) / R) / ut;
                    double vv = (t * rc + sc) / nV;
                    double qu = th + 0.5 * nu - 0.5, qv = vv + 0.5 * nv - 0.5;
                    /* detector plane of view a: u stride 1, v stride na * nu */
                    double val = orc_bilin_f(proj + a * nu, 1, na * nu, nu, nv, qu, qv, tex8);
                    vol[(z * ny + y) * nx + x] += val * t * t * scale;
                }
            }
        }
    }
    return 0;
}

/* ------------------------------------------------------------------------- */
/* 2D SART (src/CudaSartAlgorithm.cpp, cuda/2d/sart.cu)                        */
/* ------------------------------------------------------------------------- */

/* Linear interpolation of a row at index q with clamp-to-edge addressing (the
 * texture BP_SART binds with cudaAddressModeClamp, par_bp.cu:270). */
static double orc_lerp_clamp(const double *row, long n, double q, int tex8)
{
    double f = floor(q);
    long k = (long)f;
    double a = orc_frac_weight(q - f, tex8);
    long k0 = k < 0 ? 0 : (k >= n ? n - 1 : k);
    long k1 = k + 1 < 0 ? 0 : (k + 1 >= n ? n - 1 : k + 1);
    return (1.0 - a) * row[k0] + a * row[k1];
}

/*
 * SART_CUDA: `iterations` single-view steps (CCudaSartAlgorithm::run,
 * src/CudaSartAlgorithm.cpp:233-318).  Step it uses view
 * order[(iter0 + it) % norder] (sequential when order is NULL):
 *   r = (b_a - FP_a(x * mask)) * W_line[a]      FP_SART + mul_SART
 *   x += lambda * out_scale * mask * BP_SART_a(r)
 *   x = clamp(x)                                 opClampMin / opClampMax
 * W_line = opInvert(FP(mask or 1)) over all views (precomputeWeights,
 * :196-215; threshold cuda/2d/arith.cu:99-106).  BP_SART reads r with clamped
 * addressing and no adjoint weight (devBP_SART par_bp.cu:139-159 with
 * BP_SART :261-299; devFanBP_SART fan_bp.cu:164-201, constants with the
 * non-FBP scale).  kind: 3 parallel, 4 fan.  vol (float, W x H) is updated.
 */
int orc_sart2d(int kind, const float *views, long na, long ndet, long W, long H, double out_scale, int rays_per_det,
               const int *order, long norder, long iter0, long iterations, double lambda, int use_min,
               double min_value, int use_max, double max_value, int tex8, const float *sino,
               const float *vol_mask, float *vol)
{
    if (kind != 3 && kind != 4) return 1;
    const long N = W * H;
    float *src = (float *)malloc(sizeof(float) * (size_t)N);
    double *lw = (double *)malloc(sizeof(double) * (size_t)(na * ndet));
    double *row = (double *)malloc(sizeof(double) * (size_t)ndet);
    for (long i = 0; i < N; ++i) src[i] = vol_mask ? vol_mask[i] : 1.0f;
    if (kind == 3) orc_par_fp(views, na, ndet, W, H, 1.0 * out_scale, rays_per_det, tex8, src, lw);
    else orc_fan_fp(views, na, ndet, W, H, out_scale, rays_per_det, tex8, src, lw);
    for (long i = 0; i < na * ndet; ++i) {
        float v = (float)lw[i];
        lw[i] = (v > 0.000001f) ? 1.0 / (double)v : 0.0;
    }
    for (long it = 0; it < iterations; ++it) {
        long a = order ? order[(iter0 + it) % norder] : (iter0 + it) % na;
        const float *p = views + 6 * a;
        for (long i = 0; i < N; ++i) src[i] = vol_mask ? vol[i] * vol_mask[i] : vol[i];
        if (kind == 3) orc_par_fp(p, 1, ndet, W, H, out_scale, rays_per_det, tex8, src, row);
        else orc_fan_fp(p, 1, ndet, W, H, out_scale, rays_per_det, tex8, src, row);
        for (long d = 0; d < ndet; ++d) row[d] = ((double)sino[a * ndet + d] - row[d]) * lw[a * ndet + d];
        double c[6];
        if (kind == 3) {
            double dd = (double)p[4] * p[1] - (double)p[5] * p[0];
            c[0] = p[1] / dd;
            c[1] = -p[0] / dd;
            c[2] = ((double)p[3] * p[0] - (double)p[2] * p[1]) / dd;
        } else {
            double ux = p[4], uy = p[5], sx = p[0], sy = p[1], dx = p[2], dy = p[3];
            double scale = sqrt(ux * ux + uy * uy) / (ux * (sy - dy) - uy * (sx - dx));
            c[0] = scale * (sx * dy - sy * dx);
            c[1] = scale * (sy - dy);
            c[2] = -scale * (sx - dx);
            c[3] = scale * (ux * sy - uy * sx);
            c[4] = scale * uy;
            c[5] = -scale * ux;
        }
        for (long Y = 0; Y < H; ++Y) {
            for (long X = 0; X < W; ++X) {
                double x = X - 0.5 * W + 0.5, y = Y - 0.5 * H + 0.5, T;
                if (kind == 3) {
                    T = x * c[0] - y * c[1] + c[2];
                } else {
                    double yw = -y;
                    T = (c[0] + c[1] * x + c[2] * yw) / (c[3] + c[4] * x + c[5] * yw);
                }
                double u = lambda * out_scale * orc_lerp_clamp(row, ndet, T - 0.5, tex8);
                if (vol_mask) u *= vol_mask[Y * W + X];
                float nv = (float)((double)vol[Y * W + X] + u);
                if (use_min && nv < (float)min_value) nv = (float)min_value;
                if (use_max && nv > (float)max_value) nv = (float)max_value;
                vol[Y * W + X] = nv;
            }
        }
    }
    free(src);
    free(lw);
    free(row);
    return 0;
}

int orc_version(void) { return 1; }
