// Spatial taps of every FBP / FDK row filter the reference supports.
//
// The reference filters a detector row by zero-padding it to
// N = nextpow2(2 nu) samples (row at offset 0), taking a real FFT,
// multiplying by the filter's spectrum on the N / 2 + 1 bins, transforming
// back and dividing by N (cuda/3d/fdk.cu:292-398, cuda/2d/fft.cu:52-110,
// 338-595).  Because N >= 2 nu, that circular convolution equals, on the row,
// the linear convolution with the length-N inverse transform g of the
// spectrum:  y[n] = sum_k g[(n - k) mod N] x[k], |n - k| < nu.  These
// functions compute g for offsets -(nu - 1) .. nu - 1, so every filter runs
// as an exact Toeplitz product:
//   - spectral filters (Ram-Lak and its windowed forms, src/Filters.cpp:
//     131-488): the Ram-Lak spectrum (twice the real DFT of the spatial taps
//     h[0] = 1/4, h[odd i] = -1/(pi j)^2 with j = min(i, N - i),
//     src/Filters.cpp:41-69) times the window, zero beyond w = pi D;
//   - "projection" / "sinogram": the caller's real spectrum on the N / 2 + 1
//     bins, shared or one per view (fft.cu:447-496);
//   - "rprojection" / "rsinogram": the caller's spatial filter of any width W,
//     centred so that its element W / 2 sits at offset 0 (fft.cu:498-595).
// The window formulas are evaluated in single precision as the reference
// evaluates them; the ramp spectrum and the inverse transform in double.
#include "filters.h"

#include <cmath>
#include <map>
#include <mutex>

#include "b2t_internal.h"

namespace b2t {

namespace {

const float kPi = 3.14159265358979323846f;

int next_pow2(int n)
{
    int x = 1;
    while (x < n && x > 0) x *= 2;
    return x;
}

// 2 x the real DFT of the Ram-Lak spatial taps on bins 0 .. N / 2, cached per N.
const std::vector<double> &ramp_spectrum(int N)
{
    static std::mutex m;
    static std::map<int, std::vector<double>> cache;
    std::lock_guard<std::mutex> lock(m);
    auto it = cache.find(N);
    if (it != cache.end()) return it->second;
    std::vector<double> h(N, 0.0);
    h[0] = 0.25;
    for (int i = 1; i < N; i += 2) {
        const int j = (2 * i > N) ? N - i : i;
        const double f = M_PI * j;
        h[i] = -1.0 / (f * f);
    }
    std::vector<double> R(N / 2 + 1);
    for (int f = 0; f <= N / 2; ++f) {
        double s = 0.0;
        for (int i = 0; i < N; ++i) {
            if (h[i] == 0.0) continue;
            s += h[i] * std::cos(2.0 * M_PI * (double)((long long)f * i % N) / N);
        }
        R[f] = 2.0 * s;
    }
    return cache.emplace(N, std::move(R)).first->second;
}

// Window of bin f (1 <= f < F) for the spectral filter types, in float.
bool window(int32_t type, int f, int F, float w, float D, float param, float &out)
{
    const float n = (float)f;
    const float nm1 = (float)(F - 1);
    switch (type) {
    case B2T_FILTER_SHEPPLOGAN: {
        const float x = w / 2.0f / D;
        out = std::sin(x) / x;
        return true;
    }
    case B2T_FILTER_COSINE: out = std::cos(w / 2.0f / D); return true;
    case B2T_FILTER_HAMMING: out = 0.54f + 0.46f * std::cos(w / D); return true;
    case B2T_FILTER_HANN: out = (1.0f + std::cos(w / D)) / 2.0f; return true;
    case B2T_FILTER_TUKEY: {
        const float alpha = param < 0.0f ? 0.5f : param;
        const float half = (float)F / 2.0f;
        const float a = alpha * half, denom = (1.0f - alpha) * half;
        if (half - a <= n && n <= half + a) out = 1.0f;
        else out = 0.5f * (1.0f + std::cos(kPi * (n - a) / denom));
        return true;
    }
    case B2T_FILTER_LANCZOS: {
        const float x = kPi * (2.0f * n / nm1 - 1.0f);
        out = std::fabs(x) > 0.001f ? (float)std::sin(x) / x : 1.0f;
        return true;
    }
    case B2T_FILTER_TRIANGULAR: out = 2.0f / nm1 * (nm1 / 2.0f - std::fabs(n - nm1 / 2.0f)); return true;
    case B2T_FILTER_GAUSSIAN: {
        const float sigma = param < 0.0f ? 0.4f : param;
        const float q = ((float)F - 1.0f) / 2.0f;
        const float e = (n - q) / (sigma * q);
        out = std::exp(-0.5f * e * e);
        return true;
    }
    case B2T_FILTER_BARTLETTHANN:
        out = 0.62f - 0.48f * std::fabs(n / nm1 - 0.5f) - 0.38f * std::cos(2.0f * kPi * n / nm1);
        return true;
    case B2T_FILTER_BLACKMAN: {
        const float alpha = param < 0.0f ? 0.16f : param;
        out = (1.0f - alpha) / 2.0f - 0.5f * std::cos(2.0f * kPi * 0.5f * n / nm1) +
              alpha / 2.0f * std::cos(4.0f * kPi * 0.5f * n / nm1);
        return true;
    }
    case B2T_FILTER_NUTTALL:
    case B2T_FILTER_BLACKMANHARRIS:
    case B2T_FILTER_BLACKMANNUTTALL:
    case B2T_FILTER_FLATTOP: {
        // four- and five-term cosine sums a0 - a1 cos 2x + a2 cos 4x - a3 cos 6x (+ a4 cos 8x)
        static const float coef[4][5] = {{0.355768f, 0.487396f, 0.144232f, 0.012604f, 0.0f},
                                         {0.35875f, 0.48829f, 0.14128f, 0.01168f, 0.0f},
                                         {0.3635819f, 0.4891775f, 0.1365995f, 0.0106411f, 0.0f},
                                         {1.0f, 1.93f, 1.29f, 0.388f, 0.032f}};
        const int k = type == B2T_FILTER_NUTTALL ? 0 : type == B2T_FILTER_BLACKMANHARRIS ? 1
                                                   : type == B2T_FILTER_BLACKMANNUTTALL ? 2 : 3;
        const float x = kPi * n / nm1;
        const float *a = coef[k];
        out = a[0] - a[1] * std::cos(2.0f * x) + a[2] * std::cos(4.0f * x) - a[3] * std::cos(6.0f * x);
        if (k == 3) out += a[4] * std::cos(8.0f * x);
        return true;
    }
    case B2T_FILTER_KAISER: {
        const float alpha = param < 0.0f ? 3.0f : param;
        const float pa = kPi * alpha;
        const float s = 2.0f * n / nm1 - 1.0f;
        out = (float)::j0((double)(pa * std::sqrt(1.0f - s * s))) / (float)::j0((double)pa);
        return true;
    }
    case B2T_FILTER_PARZEN: {
        const float q = n / nm1;
        if (q <= 0.5f) out = 1.0f - 6.0f * q * q * (1.0f - q);
        else {
            const float c = 1.0f - q;
            out = 2.0f * c * c * c;
        }
        return true;
    }
    default: return false;
    }
}

// g[d], d = 0 .. nu-1, of the real spectrum G on bins 0 .. N/2 (Hermitian
// extension, divided by N); the taps are symmetric.
void spectrum_to_taps(const std::vector<double> &G, int N, int nu, float *g)
{
    for (int d = 0; d < nu; ++d) {
        double s = G[0] + G[N / 2] * ((d & 1) ? -1.0 : 1.0);
        for (int f = 1; f < N / 2; ++f) s += 2.0 * G[f] * std::cos(2.0 * M_PI * (double)((long long)f * d % N) / N);
        const float v = (float)(s / N);
        g[nu - 1 + d] = v;
        g[nu - 1 - d] = v;
    }
}

// g[d] of a spatial filter f of width W centred at its element W / 2 (the
// reference's placement into the length-N FFT input, fft.cu:498-525).
void spatial_to_taps(const float *f, int W, int N, int nu, float *g)
{
    std::vector<float> s(N, 0.0f);
    const int used = W < N ? W : N;
    const int start = (W - used) / 2;
    const int shift = W / 2;
    for (int i = start; i < start + used; ++i) s[(i + N - shift) % N] = f[i];
    for (int d = -(nu - 1); d < nu; ++d) g[nu - 1 + d] = s[(d + N) % N];
}

}  // namespace

bool filter_is_plain_ramlak(const b2t_filter_config *cfg)
{
    return !cfg || (cfg->type == B2T_FILTER_RAMLAK && cfg->d >= 1.0f);
}

b2t_status filter_taps(const b2t_filter_config *cfg, uint32_t nu_u, uint32_t n_views, FilterTaps &out)
{
    if (!cfg) return fail(B2T_ERR_INVALID_ARG, "filter taps: null filter");
    if (nu_u == 0 || nu_u > (1u << 20)) return fail(B2T_ERR_INVALID_ARG, "filter taps: bad row length %u", nu_u);
    const int nu = (int)nu_u;
    const int N = next_pow2(2 * nu);
    const int F = N / 2 + 1;
    const int32_t t = cfg->type;
    out.nu = nu;
    const int per_view = (t == B2T_FILTER_SINOGRAM || t == B2T_FILTER_RSINOGRAM);
    out.nsets = per_view ? (int)n_views : 1;
    out.g.assign((size_t)out.nsets * (2 * nu - 1), 0.0f);
    if (t >= B2T_FILTER_RAMLAK && t <= B2T_FILTER_PARZEN) {
        if (!(cfg->d > 0.0f)) return fail(B2T_ERR_INVALID_ARG, "filter taps: FilterD must be positive");
        const std::vector<double> &R = ramp_spectrum(N);
        std::vector<double> G(F);
        for (int f = 0; f < F; ++f) {
            const float w = kPi * 2.0f * ((float)f / (float)N);
            double v = R[f];
            float win = 1.0f;
            if (f >= 1 && t != B2T_FILTER_RAMLAK && !window(t, f, F, w, cfg->d, cfg->parameter, win))
                return fail(B2T_ERR_UNSUPPORTED, "filter taps: unknown filter type %d", t);
            v *= (double)win;
            if (w > kPi * cfg->d) v = 0.0;
            G[f] = v;
        }
        spectrum_to_taps(G, N, nu, out.g.data());
        return B2T_OK;
    }
    if (t == B2T_FILTER_PROJECTION || t == B2T_FILTER_SINOGRAM) {
        const uint32_t h = per_view ? n_views : 1;
        if (!cfg->custom || cfg->custom_width != (uint32_t)F || cfg->custom_height != h)
            return fail(B2T_ERR_INVALID_ARG, "filter size mismatch: %ux%u (received) is not %ux%d (expected)",
                        cfg->custom_height, cfg->custom_width, h, F);
        std::vector<double> G(F);
        for (int s = 0; s < out.nsets; ++s) {
            for (int f = 0; f < F; ++f) G[f] = cfg->custom[(size_t)s * F + f];
            spectrum_to_taps(G, N, nu, out.g.data() + (size_t)s * (2 * nu - 1));
        }
        return B2T_OK;
    }
    if (t == B2T_FILTER_RPROJECTION || t == B2T_FILTER_RSINOGRAM) {
        const uint32_t h = per_view ? n_views : 1;
        if (!cfg->custom || cfg->custom_width == 0 || cfg->custom_height != h)
            return fail(B2T_ERR_INVALID_ARG, "filter size mismatch: %ux%u (received) is not %uxX (expected)",
                        cfg->custom_height, cfg->custom_width, h);
        for (int s = 0; s < out.nsets; ++s)
            spatial_to_taps(cfg->custom + (size_t)s * cfg->custom_width, (int)cfg->custom_width, N, nu,
                            out.g.data() + (size_t)s * (2 * nu - 1));
        return B2T_OK;
    }
    return fail(B2T_ERR_UNSUPPORTED, "filter taps: filter type %d has no taps", t);
}

}  // namespace b2t
