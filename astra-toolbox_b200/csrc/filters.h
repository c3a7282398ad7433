// Spatial taps of the FBP / FDK row filters (filters.cpp).
#pragma once

#include <vector>

#include "b2tomo.h"

namespace b2t {

// Taps of one filter call: nsets tap sets (1, or one per view for the
// per-view "sinogram" types), each of 2 nu - 1 taps for offsets
// d = -(nu - 1) .. nu - 1 at index d + nu - 1:  y[n] = sum_k g[n - k] x[k].
struct FilterTaps {
    int nu = 0;
    int nsets = 0;
    std::vector<float> g;
    const float *set(int s) const { return g.data() + (size_t)s * (2 * nu - 1); }
};

// Ram-Lak with the default cut-off: the path that needs no tap table.
bool filter_is_plain_ramlak(const b2t_filter_config *cfg);

b2t_status filter_taps(const b2t_filter_config *cfg, uint32_t nu, uint32_t n_views, FilterTaps &out);

}  // namespace b2t
