// SIRT and CGLS reconstruction drivers (2D and 3D) behind the C ABI.
//
// Reference: CCudaSirtAlgorithm3D (src/CudaSirtAlgorithm3D.cpp:261-432),
// CCudaCglsAlgorithm3D (src/CudaCglsAlgorithm3D.cpp:264-409),
// CCudaSirtAlgorithm (src/CudaSirtAlgorithm.cpp:187-397) and
// CCudaCglsAlgorithm (src/CudaCglsAlgorithm.cpp:166-283), and
// CCudaSartAlgorithm (src/CudaSartAlgorithm.cpp:196-318; step kernels in
// sart.cu).  Same recurrences,
// same opInvert threshold (cuda/3d/arith3d.cu:87-94), same restart of CGLS at
// every run() call, same constraint and mask semantics.
//
// Differences by design:
//   - CGLS inner products and the residual norm are accumulated in FP64 (the
//     reference uses float32 dotProduct2D); alpha, beta and gamma live in
//     device memory, so an iteration issues no host synchronisation;
//   - the element-wise steps are fused: (b - A x) * W_line is one pass, the
//     update x = clamp(x + W_pix * B r) is one pass;
//   - with use_graph, one iteration is captured as a CUDA graph on the first
//     run() and replayed (the graph is rebuilt if the data pointers change).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <memory>

#include "algorithms.h"
#include "batch2d.h"
#include "arith.h"
#include "b2t_internal.h"
#include "proj2d.h"
#include "proj3d.h"
#include "sart.h"

namespace b2t {

namespace {

// ---------------------------------------------------------------------------
// fused element-wise kernels
// ---------------------------------------------------------------------------

constexpr int EW_THREADS = 256;

inline unsigned ew_blocks(size_t n)
{
    size_t b = (n + EW_THREADS - 1) / EW_THREADS;
    if (b > 148 * 32) b = 148 * 32;
    if (b < 1) b = 1;
    return (unsigned)b;
}

// r = (b - r) * w  (w may be null: weight 1; b may be null: b = 0)
__global__ void residual_weight_kernel(float *__restrict__ r, const float *__restrict__ b, const float *__restrict__ w,
                                       size_t n)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        float v = (b ? b[i] : 0.0f) - r[i];
        if (w) v *= w[i];
        r[i] = v;
    }
}

// x = clamp(x + w * d), with optional scalar and per-voxel bounds
__global__ void sirt_update_kernel(float *__restrict__ x, const float *__restrict__ w, const float *__restrict__ d,
                                   size_t n, int use_min, float vmin, int use_max, float vmax,
                                   const float *__restrict__ min_mask, const float *__restrict__ max_mask)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        float v = fmaf(w[i], d[i], x[i]);
        if (use_min && v < vmin) v = vmin;
        if (use_max && v > vmax) v = vmax;
        if (min_mask && v < min_mask[i]) v = min_mask[i];
        if (max_mask && v > max_mask[i]) v = max_mask[i];
        x[i] = v;
    }
}

// out = in * mask
__global__ void masked_copy_kernel(float *__restrict__ out, const float *__restrict__ in,
                                   const float *__restrict__ mask, size_t n)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        out[i] = in[i] * mask[i];
}

// x += sign * (s[num] / s[den]) * y   (CGLS x and r updates)
__global__ void axpy_ratio_kernel(float *__restrict__ x, const float *__restrict__ y, size_t n,
                                  const double *__restrict__ s, int num, int den, float sign)
{
    const float a = sign * (float)(s[num] / s[den]);
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        x[i] = fmaf(a, y[i], x[i]);
}

// p = z + (s[num] / s[den]) * p   (CGLS direction update)
__global__ void xpby_ratio_kernel(float *__restrict__ p, const float *__restrict__ z, size_t n,
                                  const double *__restrict__ s, int num, int den)
{
    const float beta = (float)(s[num] / s[den]);
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        p[i] = fmaf(p[i], beta, z[i]);
}

// Per-problem (segmented) forms for CGLS on a batch of problems: scalars are
// stored slot-major, s[slot * nseg + problem].  Deterministic: each chunk
// reduces in a fixed order, and each problem's chunks are summed in order.
constexpr int SEG_THREADS = 256;

__global__ void __launch_bounds__(SEG_THREADS) seg_dot_partial_kernel(const float *__restrict__ a,
                                                                       const SegChunk *__restrict__ chunks,
                                                                       double *__restrict__ partial)
{
    __shared__ double red[SEG_THREADS / 32];
    const SegChunk c = chunks[blockIdx.x];
    double acc = 0.0;
    for (int i = threadIdx.x; i < c.len; i += SEG_THREADS) {
        const double v = (double)a[c.begin + i];
        acc = fma(v, v, acc);
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < SEG_THREADS / 32; ++w) t += red[w];
        partial[blockIdx.x] = t;
    }
}

// one thread per problem: s[slot * nseg + p] = sum of its chunks' partials
__global__ void seg_dot_final_kernel(const double *__restrict__ partial, const int *__restrict__ first, int nseg,
                                     double *__restrict__ s, int slot)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= nseg) return;
    double t = 0.0;
    for (int c = first[p]; c < first[p + 1]; ++c) t += partial[c];
    s[slot * nseg + p] = t;
}

// step size of problem p; 0 when its denominator is 0 (a problem whose data
// are all zero stays at its start instead of turning into NaN)
__device__ __forceinline__ float seg_ratio(const double *s, int nseg, int num, int den, int p)
{
    const double d = s[den * nseg + p];
    return d != 0.0 ? (float)(s[num * nseg + p] / d) : 0.0f;
}

// x += sign * ratio_p * y on every chunk (chunk = one CTA)
__global__ void __launch_bounds__(SEG_THREADS) seg_axpy_ratio_kernel(float *__restrict__ x,
                                                                      const float *__restrict__ y,
                                                                      const SegChunk *__restrict__ chunks,
                                                                      const double *__restrict__ s, int nseg, int num,
                                                                      int den, float sign)
{
    const SegChunk c = chunks[blockIdx.x];
    const float a = sign * seg_ratio(s, nseg, num, den, c.seg);
    for (int i = threadIdx.x; i < c.len; i += SEG_THREADS) x[c.begin + i] = fmaf(a, y[c.begin + i], x[c.begin + i]);
}

// p = z + ratio_p * p on every chunk
__global__ void __launch_bounds__(SEG_THREADS) seg_xpby_ratio_kernel(float *__restrict__ p,
                                                                      const float *__restrict__ z,
                                                                      const SegChunk *__restrict__ chunks,
                                                                      const double *__restrict__ s, int nseg, int num,
                                                                      int den)
{
    const SegChunk c = chunks[blockIdx.x];
    const float beta = seg_ratio(s, nseg, num, den, c.seg);
    for (int i = threadIdx.x; i < c.len; i += SEG_THREADS) p[c.begin + i] = fmaf(p[c.begin + i], beta, z[c.begin + i]);
}

// ---------------------------------------------------------------------------
// operators
// ---------------------------------------------------------------------------

struct Operator {
    virtual ~Operator() = default;
    // proj (=|+=) scale * A vol
    virtual b2t_status fp(const float *vol, float *proj, float scale, int mode, cudaStream_t s) = 0;
    // vol (=|+=) scale * B proj
    virtual b2t_status bp(const float *proj, float *vol, float scale, int mode, cudaStream_t s) = 0;
    // chunk tables when the operator is a batch of independent problems
    virtual const SegTable *segments(bool vol) const { return nullptr; }
    size_t nvol = 0, nproj = 0;
};

struct Op3D : Operator {
    b2t_geom3d g;
    std::vector<b2t_view3d> views;
    b2t_params3d p;
    Op3D(const b2t_geom3d *geom, const b2t_params3d *params) : g(*geom), views(geom->views, geom->views + geom->dims.angles), p(*params)
    {
        g.views = views.data();
        nvol = (size_t)g.dims.vol_x * g.dims.vol_y * g.dims.vol_z;
        nproj = (size_t)g.dims.det_u * g.dims.angles * g.dims.det_v;
    }
    b2t_status fp(const float *vol, float *proj, float scale, int mode, cudaStream_t s) override
    {
        b2t_params3d q = p;
        q.output_scale *= scale;
        if (q.kernel != B2T_KER_MATCHED_BP) q.kernel = B2T_KER_DEFAULT;
        return fp3d_impl(&g, &q, vol, 0, proj, 0, B2T_F32, mode, s);
    }
    b2t_status bp(const float *proj, float *vol, float scale, int mode, cudaStream_t s) override
    {
        b2t_params3d q = p;
        q.output_scale *= scale;
        return bp3d_impl(&g, &q, proj, 0, vol, 0, B2T_F32, mode, s);
    }
};

// cyl_cone_vec geometry (cyl.cu): FP32, no supersampling; the BP is the
// voxel-driven one or, with B2T_KER_MATCHED_BP, the FP's transpose
struct Op3DCyl : Operator {
    b2t_geom3d_cyl g;
    std::vector<b2t_view3d_cyl> views;
    b2t_params3d p;
    Op3DCyl(const b2t_geom3d_cyl *geom, const b2t_params3d *params)
        : g(*geom), views(geom->views, geom->views + geom->dims.angles), p(*params)
    {
        g.views = views.data();
        nvol = (size_t)g.dims.vol_x * g.dims.vol_y * g.dims.vol_z;
        nproj = (size_t)g.dims.det_u * g.dims.angles * g.dims.det_v;
    }
    b2t_status fp(const float *vol, float *proj, float scale, int mode, cudaStream_t s) override
    {
        b2t_params3d q = p;
        q.output_scale *= scale;
        return fp3d_cyl_impl(&g, &q, vol, 0, proj, 0, mode, s);
    }
    b2t_status bp(const float *proj, float *vol, float scale, int mode, cudaStream_t s) override
    {
        b2t_params3d q = p;
        q.output_scale *= scale;
        return bp3d_cyl_impl(&g, &q, proj, 0, vol, 0, mode, s);
    }
};

struct Op2D : Operator {
    b2t_geom2d g;
    std::vector<b2t_view2d> views;
    uint32_t det_ss, pix_ss;
    Op2D(const b2t_geom2d *geom, uint32_t dss, uint32_t pss)
        : g(*geom), views(geom->views, geom->views + geom->dims.angles), det_ss(dss), pix_ss(pss)
    {
        g.views = views.data();
        nvol = (size_t)g.dims.vol_width * g.dims.vol_height;
        nproj = (size_t)g.dims.angles * g.dims.dets;
    }
    b2t_status fp(const float *vol, float *proj, float scale, int mode, cudaStream_t s) override
    {
        b2t_geom2d q = g;
        q.output_scale *= scale;
        return fp2d_impl(&q, det_ss, vol, 0, proj, 0, mode, s);
    }
    b2t_status bp(const float *proj, float *vol, float scale, int mode, cudaStream_t s) override
    {
        b2t_geom2d q = g;
        q.output_scale *= scale;
        return bp2d_impl(&q, pix_ss, 0, proj, 0, vol, 0, mode, s);
    }
};

// All problems of a batch (batch2d.cu) as one block-diagonal operator on the
// packed buffers: SIRT's element-wise steps then run once for the batch.
struct OpBatch2D : Operator {
    Batch2D *b;
    explicit OpBatch2D(Batch2D *batch) : b(batch)
    {
        nvol = batch->vol_total;
        nproj = batch->sino_total;
    }
    b2t_status fp(const float *vol, float *proj, float scale, int mode, cudaStream_t s) override
    {
        return batch2d_fp_impl(b, vol, proj, scale, mode, s);
    }
    b2t_status bp(const float *proj, float *vol, float scale, int mode, cudaStream_t s) override
    {
        return batch2d_bp_impl(b, proj, vol, scale, mode, s);
    }
    const SegTable *segments(bool vol) const override { return vol ? &b->vol_segs : &b->sino_segs; }
};

struct DevBuf {
    void *p = nullptr;
    ~DevBuf()
    {
        if (p) {
            cudaFree(p);
            alloc_live(-1);
        }
    }
    b2t_status alloc(size_t bytes, const char *what)
    {
        if (bytes == 0) bytes = 16;
        if (alloc_injected_failure()) return fail(B2T_ERR_NO_MEMORY, "%s: injected allocation failure", what);
        cudaError_t e = cudaMalloc(&p, bytes);
        if (e != cudaSuccess) {
            p = nullptr;
            (void)cudaGetLastError();
            return cuda_fail(e, what);
        }
        alloc_live(1);
        // zero: element-wise passes also run over the gaps between the
        // problems of a packed batch, which no projector writes
        e = cudaMemset(p, 0, bytes);
        if (e != cudaSuccess) return cuda_fail(e, what);
        return B2T_OK;
    }
    template <class T> T *as() const { return static_cast<T *>(p); }
};

}  // namespace

struct Algo {
    int type = 0;
    std::unique_ptr<Operator> op;
    b2t_algo_options opt{};
    DevBuf lineW, pixW, tmpProj, tmpVol;  // SIRT
    DevBuf r, w, p, z;                     // CGLS
    DevBuf partial, scalars;               // FP64 reductions: partials, s[0..7]
    // SART: per-view device constants, projection order, step counter, row
    DevBuf sart_par, sart_fan, sart_bpv, sart_order, sart_step, sart_r;
    int sart_norder = 0;
    int nparts_vol = 0, nparts_proj = 0;
    bool weights_ready = false;
    std::atomic<bool> abort_flag{false};
    // graph of one iteration
    cudaGraphExec_t graph = nullptr;
    const float *graph_sino = nullptr;
    float *graph_vol = nullptr;
    int graph_parity = 0;
    ~Algo()
    {
        if (graph) cudaGraphExecDestroy(graph);
    }

    size_t nv() const { return op->nvol; }
    size_t np() const { return op->nproj; }
    int nseg = 1;  // problems sharing the algorithm (a batch), one scalar set each

    enum class Space { vol, proj };

    // |a|^2 into scalar slot `slot` (per problem on a batch)
    b2t_status dot_sq(const float *a, Space sp, int slot, cudaStream_t s)
    {
        const bool is_vol = sp == Space::vol;
        const SegTable *t = op->segments(is_vol);
        if (!t) {
            const size_t n = is_vol ? nv() : np();
            const int nb = dot_num_blocks(n);
            return dot_launch(a, a, n, B2T_F32, partial.as<double>(), nb, scalars.as<double>() + slot, s);
        }
        seg_dot_partial_kernel<<<t->nchunks, SEG_THREADS, 0, s>>>(a, t->chunks, partial.as<double>());
        B2T_TRY(ew(cudaGetLastError(), "batch dot partials"));
        seg_dot_final_kernel<<<(t->nseg + 127) / 128, 128, 0, s>>>(partial.as<double>(), t->first, t->nseg,
                                                                   scalars.as<double>(), slot);
        return ew(cudaGetLastError(), "batch dot final");
    }

    // x += sign * (s[num] / s[den]) * y over a volume or projection buffer
    b2t_status axpy_ratio(float *x, const float *y, Space sp, int num, int den, float sign, cudaStream_t s)
    {
        const bool is_vol = sp == Space::vol;
        const SegTable *t = op->segments(is_vol);
        if (!t) {
            const size_t n = is_vol ? nv() : np();
            axpy_ratio_kernel<<<ew_blocks(n), EW_THREADS, 0, s>>>(x, y, n, scalars.as<double>(), num, den, sign);
        } else {
            seg_axpy_ratio_kernel<<<t->nchunks, SEG_THREADS, 0, s>>>(x, y, t->chunks, scalars.as<double>(), t->nseg,
                                                                     num, den, sign);
        }
        return ew(cudaGetLastError(), "CGLS axpy");
    }

    // p = z + (s[num] / s[den]) * p over the volume
    b2t_status xpby_ratio(float *p_, const float *z_, int num, int den, cudaStream_t s)
    {
        const SegTable *t = op->segments(true);
        if (!t) {
            xpby_ratio_kernel<<<ew_blocks(nv()), EW_THREADS, 0, s>>>(p_, z_, nv(), scalars.as<double>(), num, den);
        } else {
            seg_xpby_ratio_kernel<<<t->nchunks, SEG_THREADS, 0, s>>>(p_, z_, t->chunks, scalars.as<double>(), t->nseg,
                                                                     num, den);
        }
        return ew(cudaGetLastError(), "CGLS p update");
    }

    b2t_status ew(cudaError_t e, const char *what)
    {
        count_launches(1);
        if (e != cudaSuccess) return cuda_fail(e, what);
        return B2T_OK;
    }

    // SIRT line / pixel weights (precomputeWeights, CudaSirtAlgorithm3D.cpp:261-296)
    b2t_status sirt_weights(cudaStream_t s)
    {
        const float *vm = opt.vol_mask, *sm = opt.sino_mask;
        if (vm) {
            B2T_TRY(op->fp(vm, lineW.as<float>(), 1.0f, B2T_MODE_SET, s));
        } else {
            B2T_TRY(vec_op_impl(B2T_OP_SET, tmpVol.as<float>(), nullptr, nullptr, 1.0f, nv(), s));
            B2T_TRY(op->fp(tmpVol.as<float>(), lineW.as<float>(), 1.0f, B2T_MODE_SET, s));
        }
        B2T_TRY(vec_op_impl(B2T_OP_INVERT, lineW.as<float>(), nullptr, nullptr, 0.0f, np(), s));
        if (sm) B2T_TRY(vec_op_impl(B2T_OP_MUL, lineW.as<float>(), sm, nullptr, 0.0f, np(), s));
        if (sm) {
            B2T_TRY(op->bp(sm, pixW.as<float>(), 1.0f, B2T_MODE_SET, s));
        } else {
            B2T_TRY(vec_op_impl(B2T_OP_SET, tmpProj.as<float>(), nullptr, nullptr, 1.0f, np(), s));
            B2T_TRY(op->bp(tmpProj.as<float>(), pixW.as<float>(), 1.0f, B2T_MODE_SET, s));
        }
        B2T_TRY(vec_op_impl(B2T_OP_INVERT, pixW.as<float>(), nullptr, nullptr, 0.0f, nv(), s));
        if (vm) B2T_TRY(vec_op_impl(B2T_OP_MUL, pixW.as<float>(), vm, nullptr, 0.0f, nv(), s));
        B2T_TRY(vec_op_impl(B2T_OP_MUL_SCALAR, pixW.as<float>(), nullptr, nullptr, opt.relaxation, nv(), s));
        return B2T_OK;
    }

    // vol to project: x, or x * mask in tmp
    const float *masked(const float *x, float *tmp, cudaStream_t s, b2t_status &st)
    {
        st = B2T_OK;
        if (!opt.vol_mask) return x;
        masked_copy_kernel<<<ew_blocks(nv()), EW_THREADS, 0, s>>>(tmp, x, opt.vol_mask, nv());
        st = ew(cudaGetLastError(), "masked copy");
        return tmp;
    }

    b2t_status sirt_iteration(const float *sino, float *vol, cudaStream_t s)
    {
        b2t_status st;
        const float *xv = masked(vol, tmpVol.as<float>(), s, st);
        B2T_TRY(st);
        B2T_TRY(op->fp(xv, tmpProj.as<float>(), 1.0f, B2T_MODE_SET, s));
        residual_weight_kernel<<<ew_blocks(np()), EW_THREADS, 0, s>>>(tmpProj.as<float>(), sino, lineW.as<float>(), np());
        B2T_TRY(ew(cudaGetLastError(), "SIRT residual"));
        B2T_TRY(op->bp(tmpProj.as<float>(), tmpVol.as<float>(), 1.0f, B2T_MODE_SET, s));
        sirt_update_kernel<<<ew_blocks(nv()), EW_THREADS, 0, s>>>(
            vol, pixW.as<float>(), tmpVol.as<float>(), nv(), opt.use_min, opt.min_value, opt.use_max, opt.max_value,
            opt.min_mask, opt.max_mask);
        return ew(cudaGetLastError(), "SIRT update");
    }

    // CGLS restart (CudaCglsAlgorithm3D.cpp:295-316): r = b - A x, p = B r, gamma = |p|^2
    b2t_status cgls_restart(const float *sino, float *vol, cudaStream_t s)
    {
        b2t_status st;
        const float *xv = masked(vol, z.as<float>(), s, st);
        B2T_TRY(st);
        B2T_TRY(op->fp(xv, r.as<float>(), 1.0f, B2T_MODE_SET, s));
        residual_weight_kernel<<<ew_blocks(np()), EW_THREADS, 0, s>>>(r.as<float>(), sino, nullptr, np());
        B2T_TRY(ew(cudaGetLastError(), "CGLS residual"));
        B2T_TRY(op->bp(r.as<float>(), p.as<float>(), 1.0f, B2T_MODE_SET, s));
        if (opt.vol_mask) B2T_TRY(vec_op_impl(B2T_OP_MUL, p.as<float>(), opt.vol_mask, nullptr, 0.0f, nv(), s));
        return dot_sq(p.as<float>(), Space::vol, 0, s);  // gamma in slot 0
    }

    // one CGLS iteration; gamma in slot g, new gamma into slot 1 - g; ww in slot 2
    b2t_status cgls_iteration(float *vol, int g, cudaStream_t s)
    {
        B2T_TRY(op->fp(p.as<float>(), w.as<float>(), 1.0f, B2T_MODE_SET, s));
        B2T_TRY(dot_sq(w.as<float>(), Space::proj, 2, s));
        B2T_TRY(axpy_ratio(vol, p.as<float>(), Space::vol, g, 2, 1.0f, s));
        B2T_TRY(axpy_ratio(r.as<float>(), w.as<float>(), Space::proj, g, 2, -1.0f, s));
        B2T_TRY(op->bp(r.as<float>(), z.as<float>(), 1.0f, B2T_MODE_SET, s));
        if (opt.vol_mask) B2T_TRY(vec_op_impl(B2T_OP_MUL, z.as<float>(), opt.vol_mask, nullptr, 0.0f, nv(), s));
        B2T_TRY(dot_sq(z.as<float>(), Space::vol, 1 - g, s));
        return xpby_ratio(p.as<float>(), z.as<float>(), 1 - g, g, s);
    }

    // SART line weights: W_line = opInvert(FP(mask or 1)) (precomputeWeights,
    // CudaSartAlgorithm.cpp:196-215); no pixel weights
    b2t_status sart_weights(cudaStream_t s)
    {
        const float *vm = opt.vol_mask;
        if (vm) {
            B2T_TRY(op->fp(vm, lineW.as<float>(), 1.0f, B2T_MODE_SET, s));
        } else {
            B2T_TRY(vec_op_impl(B2T_OP_SET, tmpVol.as<float>(), nullptr, nullptr, 1.0f, nv(), s));
            B2T_TRY(op->fp(tmpVol.as<float>(), lineW.as<float>(), 1.0f, B2T_MODE_SET, s));
        }
        return vec_op_impl(B2T_OP_INVERT, lineW.as<float>(), nullptr, nullptr, 0.0f, np(), s);
    }

    // one SART step: the view of the current step, then advance the counter
    b2t_status sart_iteration(const float *sino, float *vol, cudaStream_t s)
    {
        const Op2D *o = static_cast<const Op2D *>(op.get());
        const b2t_dims2d &d = o->g.dims;
        b2t_status st;
        const float *xv = masked(vol, tmpVol.as<float>(), s, st);
        B2T_TRY(st);
        SartResidualLaunch R;
        R.vol = xv;
        R.vol_pitch = d.vol_width;
        R.sino = sino;
        R.line_weight = lineW.as<float>();
        R.r = sart_r.as<float>();
        R.W = d.vol_width;
        R.H = d.vol_height;
        R.ndet = d.dets;
        R.rays = (int)o->det_ss;
        R.kind = o->g.kind;
        R.out_scale = o->g.output_scale;
        R.par = sart_par.as<ParFPView>();
        R.fan = sart_fan.as<b2t_view2d>();
        R.order = sart_order.as<int>();
        R.norder = sart_norder;
        R.step = sart_step.as<long long>();
        B2T_TRY(sart_residual_launch(R, s));
        SartUpdateLaunch U;
        U.vol = vol;
        U.vol_pitch = d.vol_width;
        U.r = sart_r.as<float>();
        U.mask = opt.vol_mask;
        U.W = d.vol_width;
        U.H = d.vol_height;
        U.ndet = d.dets;
        U.kind = o->g.kind;
        U.scale = opt.relaxation * o->g.output_scale;
        U.use_min = opt.use_min;
        U.use_max = opt.use_max;
        U.min_value = opt.min_value;
        U.max_value = opt.max_value;
        U.views = sart_bpv.as<BPView2D>();
        U.order = sart_order.as<int>();
        U.norder = sart_norder;
        U.step = sart_step.as<long long>();
        B2T_TRY(sart_update_launch(U, s));
        return sart_advance_launch(sart_step.as<long long>(), s);
    }

    b2t_status iteration(const float *sino, float *vol, int parity, cudaStream_t s)
    {
        if (type == B2T_ALGO_SIRT) return sirt_iteration(sino, vol, s);
        if (type == B2T_ALGO_SART) return sart_iteration(sino, vol, s);
        return cgls_iteration(vol, parity, s);
    }
};

b2t_status algo_create(int32_t type, Operator *op_raw, const b2t_algo_options *opt, b2t_algo **out)
{
    std::unique_ptr<Operator> op(op_raw);
    if (!out) return fail(B2T_ERR_INVALID_ARG, "b2t_algo_create: null output");
    *out = nullptr;
    if (type != B2T_ALGO_SIRT && type != B2T_ALGO_CGLS && type != B2T_ALGO_SART)
        return fail(B2T_ERR_INVALID_ARG, "b2t_algo_create: unknown algorithm type %d", type);
    std::unique_ptr<Algo> a(new Algo);
    a->type = type;
    a->op = std::move(op);
    if (opt) a->opt = *opt;
    else {
        a->opt.relaxation = 1.0f;
    }
    const size_t vb = a->nv() * sizeof(float), pb = a->np() * sizeof(float);
    if (type == B2T_ALGO_SART) {
        B2T_TRY(a->lineW.alloc(pb, "SART line weights"));
        B2T_TRY(a->tmpVol.alloc(vb, "SART volume buffer"));
    } else if (type == B2T_ALGO_SIRT) {
        B2T_TRY(a->lineW.alloc(pb, "SIRT line weights"));
        B2T_TRY(a->pixW.alloc(vb, "SIRT pixel weights"));
        B2T_TRY(a->tmpProj.alloc(pb, "SIRT projection buffer"));
        B2T_TRY(a->tmpVol.alloc(vb, "SIRT volume buffer"));
    } else {
        B2T_TRY(a->r.alloc(pb, "CGLS r"));
        B2T_TRY(a->w.alloc(pb, "CGLS w"));
        B2T_TRY(a->p.alloc(vb, "CGLS p"));
        B2T_TRY(a->z.alloc(vb, "CGLS z"));
        B2T_TRY(a->tmpProj.alloc(pb, "residual buffer"));
    }
    if (!a->tmpProj.p) B2T_TRY(a->tmpProj.alloc(pb, "residual buffer"));
    const SegTable *tv = a->op->segments(true), *tp = a->op->segments(false);
    size_t nparts = DOT_MAX_BLOCKS;
    if (tv) {
        a->nseg = tv->nseg;
        nparts = std::max<size_t>(nparts, (size_t)std::max(tv->nchunks, tp->nchunks));
    }
    B2T_TRY(a->partial.alloc(sizeof(double) * nparts, "dot partials"));
    B2T_TRY(a->scalars.alloc(sizeof(double) * 8 * a->nseg, "CGLS scalars"));
    *out = reinterpret_cast<b2t_algo *>(a.release());
    return B2T_OK;
}

b2t_status algo_create3d_impl(int32_t type, const b2t_geom3d *geom, const b2t_params3d *params,
                              const b2t_algo_options *opt, b2t_algo **out)
{
    if (type == B2T_ALGO_SART) return fail(B2T_ERR_INVALID_ARG, "b2t_algo_create3d: SART is 2D only");
    B2T_TRY(validate3d(geom, "b2t_algo_create3d"));
    if (!params) return fail(B2T_ERR_INVALID_ARG, "b2t_algo_create3d: null params");
    return algo_create(type, new Op3D(geom, params), opt, out);
}

// Device tables of SART: per-view FP and BP_SART constants, the sequential
// projection order, the step counter (CudaSartAlgorithm.cpp:67-110).
static b2t_status sart_setup(Algo *a, const Op2D *o)
{
    const b2t_dims2d &d = o->g.dims;
    const uint32_t na = d.angles;
    std::vector<ParFPView> par(na);
    std::vector<BPView2D> bpv(na);
    std::vector<int> order(na);
    for (uint32_t i = 0; i < na; ++i) {
        if (o->g.kind == B2T_GEOM_PAR2D) par_fp_view(o->g.views[i], d, o->g.output_scale, par[i]);
        bp2d_view(o->g.kind, 0, o->g.views[i], bpv[i]);
        order[i] = (int)i;
    }
    B2T_TRY(a->sart_par.alloc(sizeof(ParFPView) * na, "SART view table"));
    B2T_TRY(a->sart_fan.alloc(sizeof(b2t_view2d) * na, "SART view table"));
    B2T_TRY(a->sart_bpv.alloc(sizeof(BPView2D) * na, "SART view table"));
    B2T_TRY(a->sart_order.alloc(sizeof(int) * na, "SART projection order"));
    B2T_TRY(a->sart_step.alloc(sizeof(long long), "SART step counter"));
    B2T_TRY(a->sart_r.alloc(sizeof(float) * d.dets, "SART residual row"));
    B2T_CUDA_TRY(cudaMemcpy(a->sart_par.p, par.data(), sizeof(ParFPView) * na, cudaMemcpyHostToDevice), "SART upload");
    B2T_CUDA_TRY(cudaMemcpy(a->sart_fan.p, o->g.views, sizeof(b2t_view2d) * na, cudaMemcpyHostToDevice), "SART upload");
    B2T_CUDA_TRY(cudaMemcpy(a->sart_bpv.p, bpv.data(), sizeof(BPView2D) * na, cudaMemcpyHostToDevice), "SART upload");
    B2T_CUDA_TRY(cudaMemcpy(a->sart_order.p, order.data(), sizeof(int) * na, cudaMemcpyHostToDevice), "SART upload");
    a->sart_norder = (int)na;
    return B2T_OK;
}

b2t_status algo_create3d_cyl_impl(int32_t type, const b2t_geom3d_cyl *geom, const b2t_params3d *params,
                                  const b2t_algo_options *opt, b2t_algo **out)
{
    if (!geom || !geom->views || !params) return fail(B2T_ERR_INVALID_ARG, "b2t_algo_create3d_cyl: null argument");
    if (type == B2T_ALGO_SART) return fail(B2T_ERR_INVALID_ARG, "b2t_algo_create3d_cyl: SART is 2D only");
    if (params->det_supersample > 1 || params->voxel_supersample > 1)
        return fail(B2T_ERR_UNSUPPORTED,
                    "Detector/voxel supersampling is not supported for cyl_cone_vec geometry.");
    return algo_create(type, new Op3DCyl(geom, params), opt, out);
}

b2t_status algo_create2d_impl(int32_t type, const b2t_geom2d *geom, uint32_t det_ss, uint32_t pix_ss,
                              const b2t_algo_options *opt, b2t_algo **out)
{
    B2T_TRY(validate2d(geom, "b2t_algo_create2d"));
    if (type == B2T_ALGO_SART) {
        if (pix_ss > 1) return fail(B2T_ERR_UNSUPPORTED, "SART_CUDA: no pixel supersampling (BP_SART, par_bp.cu:265)");
        if (opt && opt->sino_mask)
            return fail(B2T_ERR_UNSUPPORTED, "SART_CUDA: Sinogram mask option is not supported");
        if (opt && (opt->min_mask || opt->max_mask))
            return fail(B2T_ERR_UNSUPPORTED, "SART_CUDA: per-pixel bounds are not supported");
    }
    B2T_TRY(algo_create(type, new Op2D(geom, det_ss ? det_ss : 1, pix_ss ? pix_ss : 1), opt, out));
    if (type == B2T_ALGO_SART) {
        Algo *a = reinterpret_cast<Algo *>(*out);
        const b2t_status st = sart_setup(a, static_cast<const Op2D *>(a->op.get()));
        if (st != B2T_OK) {
            delete a;
            *out = nullptr;
            return st;
        }
    }
    return B2T_OK;
}

b2t_status algo_set_order_impl(b2t_algo *h, const int32_t *order, uint32_t n)
{
    Algo *a = reinterpret_cast<Algo *>(h);
    if (!a || !order || n == 0) return fail(B2T_ERR_INVALID_ARG, "b2t_algo_set_projection_order: null or empty order");
    if (a->type != B2T_ALGO_SART)
        return fail(B2T_ERR_INVALID_ARG, "b2t_algo_set_projection_order: the algorithm is not SART");
    const uint32_t na = static_cast<const Op2D *>(a->op.get())->g.dims.angles;
    for (uint32_t i = 0; i < n; ++i)
        if (order[i] < 0 || (uint32_t)order[i] >= na)
            return fail(B2T_ERR_INVALID_ARG, "b2t_algo_set_projection_order: view %d outside 0..%u", order[i], na - 1);
    DevBuf nb;
    B2T_TRY(nb.alloc(sizeof(int) * n, "SART projection order"));
    B2T_CUDA_TRY(cudaMemcpy(nb.p, order, sizeof(int) * n, cudaMemcpyHostToDevice), "SART order upload");
    std::swap(a->sart_order.p, nb.p);
    a->sart_norder = (int)n;
    if (a->graph) {  // the captured step holds the old order's address
        cudaGraphExecDestroy(a->graph);
        a->graph = nullptr;
    }
    return B2T_OK;
}

b2t_status algo_create_batch2d_impl(int32_t type, Batch2D *batch, const b2t_algo_options *opt, b2t_algo **out)
{
    if (!batch) return fail(B2T_ERR_INVALID_ARG, "b2t_algo_create_batch2d: null batch");
    if (opt && (opt->vol_mask || opt->sino_mask || opt->min_mask || opt->max_mask))
        return fail(B2T_ERR_UNSUPPORTED, "b2t_algo_create_batch2d: masks are not supported on a batch");
    return algo_create(type, new OpBatch2D(batch), opt, out);
}

b2t_status algo_run_impl(b2t_algo *h, const float *sino, float *vol, int32_t iters, int32_t use_graph, cudaStream_t s)
{
    Algo *a = reinterpret_cast<Algo *>(h);
    if (!a || !sino || !vol) return fail(B2T_ERR_INVALID_ARG, "b2t_algo_run: null argument");
    if (iters < 0) return fail(B2T_ERR_INVALID_ARG, "b2t_algo_run: negative iteration count");
    a->abort_flag.store(false);
    if (a->type == B2T_ALGO_SIRT) {
        // masks change the weights: recompute them every run (CudaSirtAlgorithm3D.cpp:340-341)
        if (!a->weights_ready || a->opt.vol_mask || a->opt.sino_mask) {
            B2T_TRY(a->sirt_weights(s));
            a->weights_ready = true;
        }
    } else if (a->type == B2T_ALGO_SART) {
        // with a mask the weights follow it every run (CudaSartAlgorithm.cpp:265-269)
        if (!a->weights_ready || a->opt.vol_mask) {
            B2T_TRY(a->sart_weights(s));
            a->weights_ready = true;
        }
    } else {
        B2T_TRY(a->cgls_restart(sino, vol, s));
    }
    if (iters == 0) return B2T_OK;

    if (use_graph) {
        // capture one iteration per parity (SIRT has one shape; CGLS alternates
        // the gamma slots, so two iterations are captured as one graph)
        const int per_graph = (a->type == B2T_ALGO_CGLS) ? 2 : 1;
        if (!a->graph || a->graph_sino != sino || a->graph_vol != vol) {
            if (a->graph) {
                cudaGraphExecDestroy(a->graph);
                a->graph = nullptr;
            }
            cudaStream_t cs;
            B2T_CUDA_TRY(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking), "graph capture stream");
            cudaGraph_t g = nullptr;
            b2t_status st = B2T_OK;
            cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
            if (e == cudaSuccess) {
                for (int k = 0; k < per_graph && st == B2T_OK; ++k) st = a->iteration(sino, vol, k, cs);
                cudaError_t e2 = cudaStreamEndCapture(cs, &g);
                if (st == B2T_OK && e2 != cudaSuccess) st = cuda_fail(e2, "end graph capture");
            } else {
                st = cuda_fail(e, "begin graph capture");
            }
            if (st == B2T_OK) {
                e = cudaGraphInstantiate(&a->graph, g, 0);
                if (e != cudaSuccess) st = cuda_fail(e, "graph instantiate");
            }
            if (g) cudaGraphDestroy(g);
            cudaStreamDestroy(cs);
            B2T_TRY(st);
            a->graph_sino = sino;
            a->graph_vol = vol;
        }
        int done = 0;
        while (done + per_graph <= iters) {
            if (a->abort_flag.load()) return fail(B2T_ERR_ABORTED, "b2t_algo_run: aborted after %d iterations", done);
            B2T_CUDA_TRY(cudaGraphLaunch(a->graph, s), "graph launch");
            count_launches(1);
            done += per_graph;
        }
        for (; done < iters; ++done) B2T_TRY(a->iteration(sino, vol, done & 1, s));
        return B2T_OK;
    }
    for (int it = 0; it < iters; ++it) {
        if (a->abort_flag.load()) return fail(B2T_ERR_ABORTED, "b2t_algo_run: aborted after %d iterations", it);
        B2T_TRY(a->iteration(sino, vol, it & 1, s));
    }
    return B2T_OK;
}

b2t_status algo_residual_impl(b2t_algo *h, const float *sino, const float *vol, double *norm, cudaStream_t s)
{
    Algo *a = reinterpret_cast<Algo *>(h);
    if (!a || !sino || !vol || !norm) return fail(B2T_ERR_INVALID_ARG, "b2t_algo_residual_norm: null argument");
    float *tp = a->tmpProj.as<float>();
    b2t_status st;
    float *tv = (a->type == B2T_ALGO_CGLS) ? a->z.as<float>() : a->tmpVol.as<float>();
    const float *xv = a->masked(vol, tv, s, st);
    B2T_TRY(st);
    B2T_TRY(a->op->fp(xv, tp, 1.0f, B2T_MODE_SET, s));
    residual_weight_kernel<<<ew_blocks(a->np()), EW_THREADS, 0, s>>>(tp, sino, nullptr, a->np());
    B2T_TRY(a->ew(cudaGetLastError(), "residual"));
    // one norm over the whole buffer (every problem of a batch), in the last
    // scalar slot
    double *slot = a->scalars.as<double>() + 7 * a->nseg;
    B2T_TRY(dot_launch(tp, tp, a->np(), B2T_F32, a->partial.as<double>(), dot_num_blocks(a->np()), slot, s));
    double v = 0.0;
    B2T_CUDA_TRY(cudaMemcpyAsync(&v, slot, sizeof(double), cudaMemcpyDeviceToHost, s), "residual readback");
    B2T_CUDA_TRY(cudaStreamSynchronize(s), "residual synchronize");
    *norm = std::sqrt(v);
    return B2T_OK;
}

void algo_abort_impl(b2t_algo *h)
{
    Algo *a = reinterpret_cast<Algo *>(h);
    if (a) a->abort_flag.store(true);
}

void algo_destroy_impl(b2t_algo *h) { delete reinterpret_cast<Algo *>(h); }

}  // namespace b2t
