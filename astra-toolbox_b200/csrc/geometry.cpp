// Host-side geometry conversion: projection-geometry parameters -> per-view
// vectors, and normalisation to unit voxels centred on the origin.
//
// These follow the reference's arithmetic operation by operation (double
// vectors built from float32 geometry parameters, float window centre and
// inverse voxel size) so that the per-view vectors are bit-identical to what
// the reference feeds its kernels:
//   genConeProjections / genPar3DProjections  src/GeometryUtil3D.cpp:42-172
//   convertAstraGeometry_internal             src/GeometryUtil3D.cpp:569-593
//   genParProjections / genFanProjections     src/GeometryUtil2D.cpp:40-104
//   convertAstraGeometry_internal (2D)        src/GeometryUtil2D.cpp:182-209
// The tests compare them against the reference's own GeometryUtil build.
#include <cmath>
#include <cstring>

#include "b2t_internal.h"

using namespace b2t;

namespace {

struct V3 {
    double x, y, z;
};

// Rotation about z by alpha (promoted float angle), the ROTATE0 macro of
// src/GeometryUtil3D.cpp:66.
inline V3 rot_z(const V3 &b, double alpha)
{
    V3 r;
    r.x = b.x * cos(alpha) - b.y * sin(alpha);
    r.y = b.x * sin(alpha) + b.y * cos(alpha);
    r.z = b.z;
    return r;
}

inline void put(double *dst, const V3 &v)
{
    dst[0] = v.x;
    dst[1] = v.y;
    dst[2] = v.z;
}

}  // namespace

extern "C" b2t_status b2t_cone_views(uint32_t n_angles, uint32_t det_cols, uint32_t det_rows,
                                     float src_origin, float origin_det, float det_spacing_x,
                                     float det_spacing_y, const float *angles, b2t_view3d *out)
{
    clear_error();
    if (!angles || !out) return fail(B2T_ERR_INVALID_ARG, "b2t_cone_views: null pointer");
    const double fOriginSourceDistance = src_origin, fOriginDetectorDistance = origin_det;
    const double fDetUSize = det_spacing_x, fDetVSize = det_spacing_y;
    V3 src{0.0f, -fOriginSourceDistance, 0.0f};
    V3 dets{det_cols * fDetUSize * -0.5f, fOriginDetectorDistance, det_rows * fDetVSize * -0.5f};
    V3 detu{fDetUSize, 0.0f, 0.0f};
    V3 detv{0.0f, 0.0f, fDetVSize};
    for (uint32_t i = 0; i < n_angles; ++i) {
        double a = angles[i];
        put(out[i].src, rot_z(src, a));
        put(out[i].det_s, rot_z(dets, a));
        put(out[i].det_u, rot_z(detu, a));
        put(out[i].det_v, rot_z(detv, a));
    }
    return B2T_OK;
}

extern "C" b2t_status b2t_par3d_views(uint32_t n_angles, uint32_t det_cols, uint32_t det_rows,
                                      float det_spacing_x, float det_spacing_y, const float *angles,
                                      b2t_view3d *out)
{
    clear_error();
    if (!angles || !out) return fail(B2T_ERR_INVALID_ARG, "b2t_par3d_views: null pointer");
    const double fDetUSize = det_spacing_x, fDetVSize = det_spacing_y;
    V3 ray{0.0f, 1.0f, 0.0f};
    V3 dets{det_cols * fDetUSize * -0.5f, 0.0f, det_rows * fDetVSize * -0.5f};
    V3 detu{fDetUSize, 0.0f, 0.0f};
    V3 detv{0.0f, 0.0f, fDetVSize};
    for (uint32_t i = 0; i < n_angles; ++i) {
        double a = angles[i];
        put(out[i].src, rot_z(ray, a));
        put(out[i].det_s, rot_z(dets, a));
        put(out[i].det_u, rot_z(detu, a));
        put(out[i].det_v, rot_z(detv, a));
    }
    return B2T_OK;
}

extern "C" b2t_status b2t_vec_views3d(uint32_t n_angles, uint32_t det_cols, uint32_t det_rows,
                                      const double *data, b2t_view3d *out)
{
    clear_error();
    if (!data || !out) return fail(B2T_ERR_INVALID_ARG, "b2t_vec_views3d: null pointer");
    for (uint32_t i = 0; i < n_angles; ++i) {
        const double *d = data + 12 * (size_t)i;
        b2t_view3d &p = out[i];
        p.src[0] = d[0];
        p.src[1] = d[1];
        p.src[2] = d[2];
        p.det_u[0] = d[6];
        p.det_u[1] = d[7];
        p.det_u[2] = d[8];
        p.det_v[0] = d[9];
        p.det_v[1] = d[10];
        p.det_v[2] = d[11];
        // centre -> corner, as the vec geometry classes convert it
        for (int k = 0; k < 3; ++k)
            p.det_s[k] = d[3 + k] - 0.5 * det_rows * p.det_v[k] - 0.5 * det_cols * p.det_u[k];
    }
    return B2T_OK;
}

extern "C" b2t_status b2t_normalize_views3d(const b2t_volgeom3d *vol, int32_t kind, uint32_t n,
                                            b2t_view3d *views, float *vol_scale_out)
{
    clear_error();
    if (!vol || !views || !vol_scale_out)
        return fail(B2T_ERR_INVALID_ARG, "b2t_normalize_views3d: null pointer");
    if (kind != B2T_GEOM_CONE && kind != B2T_GEOM_PAR3D)
        return fail(B2T_ERR_INVALID_ARG, "b2t_normalize_views3d: kind must be PAR3D or CONE");
    if (vol->cols == 0 || vol->rows == 0 || vol->slices == 0)
        return fail(B2T_ERR_INVALID_ARG, "b2t_normalize_views3d: empty volume");
    // CVolumeGeometry3D dependent quantities (float32, src/VolumeGeometry3D.cpp:161-170)
    float lenX = vol->max_x - vol->min_x;
    float lenY = vol->max_y - vol->min_y;
    float lenZ = vol->max_z - vol->min_z;
    float pixX = lenX / (float)vol->cols;
    float pixY = lenY / (float)vol->rows;
    float pixZ = lenZ / (float)vol->slices;
    if (!(pixX > 0.0f) || !(pixY > 0.0f) || !(pixZ > 0.0f))
        return fail(B2T_ERR_INVALID_ARG, "b2t_normalize_views3d: window min must be below max");
    float dx = -(vol->min_x + vol->max_x) / 2;
    float dy = -(vol->min_y + vol->max_y) / 2;
    float dz = -(vol->min_z + vol->max_z) / 2;
    float fx = 1.0f / pixX;
    float fy = 1.0f / pixY;
    float fz = 1.0f / pixZ;
    for (uint32_t i = 0; i < n; ++i) {
        b2t_view3d &p = views[i];
        // translate (cone: source and detector; parallel: detector only)
        if (kind == B2T_GEOM_CONE) {
            p.src[0] += dx;
            p.src[1] += dy;
            p.src[2] += dz;
        }
        p.det_s[0] += dx;
        p.det_s[1] += dy;
        p.det_s[2] += dz;
        // scale every vector
        double *vecs[4] = {p.src, p.det_s, p.det_u, p.det_v};
        for (double *v : vecs) {
            v[0] *= fx;
            v[1] *= fy;
            v[2] *= fz;
        }
    }
    vol_scale_out[0] = pixX;
    vol_scale_out[1] = pixY;
    vol_scale_out[2] = pixZ;
    return B2T_OK;
}

// convertAstraGeometry_unscaled_internal (src/GeometryUtil3D.cpp:597-617):
// the cylindrical-detector views are translated (source and detector centre)
// but not scaled; the voxel size travels separately.
extern "C" b2t_status b2t_normalize_views3d_cyl(const b2t_volgeom3d *vol, uint32_t n, b2t_view3d_cyl *views,
                                                float *vol_scale_out)
{
    clear_error();
    if (!vol || !views || !vol_scale_out) return fail(B2T_ERR_INVALID_ARG, "b2t_normalize_views3d_cyl: null pointer");
    if (vol->cols == 0 || vol->rows == 0 || vol->slices == 0)
        return fail(B2T_ERR_INVALID_ARG, "b2t_normalize_views3d_cyl: empty volume");
    float pixX = (vol->max_x - vol->min_x) / (float)vol->cols;
    float pixY = (vol->max_y - vol->min_y) / (float)vol->rows;
    float pixZ = (vol->max_z - vol->min_z) / (float)vol->slices;
    if (!(pixX > 0.0f) || !(pixY > 0.0f) || !(pixZ > 0.0f))
        return fail(B2T_ERR_INVALID_ARG, "b2t_normalize_views3d_cyl: window min must be below max");
    float dx = -(vol->min_x + vol->max_x) / 2;
    float dy = -(vol->min_y + vol->max_y) / 2;
    float dz = -(vol->min_z + vol->max_z) / 2;
    for (uint32_t i = 0; i < n; ++i) {
        b2t_view3d_cyl &p = views[i];
        if (!(p.radius > 0.0)) return fail(B2T_ERR_INVALID_ARG, "b2t_normalize_views3d_cyl: radius must be > 0");
        p.src[0] += dx;
        p.src[1] += dy;
        p.src[2] += dz;
        p.det_c[0] += dx;
        p.det_c[1] += dy;
        p.det_c[2] += dz;
    }
    vol_scale_out[0] = pixX;
    vol_scale_out[1] = pixY;
    vol_scale_out[2] = pixZ;
    return B2T_OK;
}

// ---------------------------------------------------------------------------
// 2D
// ---------------------------------------------------------------------------

extern "C" b2t_status b2t_par_views(uint32_t n_angles, uint32_t n_dets, float det_width,
                                    const float *angles, b2t_view2d *out)
{
    clear_error();
    if (!angles || !out) return fail(B2T_ERR_INVALID_ARG, "b2t_par_views: null pointer");
    const double fDetSize = det_width;
    // SParProjection fields are float (src/GeometryUtil2D.cpp:40-78)
    float rx0 = 0.0f, ry0 = 1.0f;
    float sx0 = (float)(n_dets * fDetSize * -0.5f), sy0 = 0.0f;
    float ux0 = (float)fDetSize, uy0 = 0.0f;
    for (uint32_t i = 0; i < n_angles; ++i) {
        double a = angles[i];
        b2t_view2d &p = out[i];
        p.src[0] = (float)(rx0 * cos(a) - ry0 * sin(a));
        p.src[1] = (float)(rx0 * sin(a) + ry0 * cos(a));
        p.det_s[0] = (float)(sx0 * cos(a) - sy0 * sin(a));
        p.det_s[1] = (float)(sx0 * sin(a) + sy0 * cos(a));
        p.det_u[0] = (float)(ux0 * cos(a) - uy0 * sin(a));
        p.det_u[1] = (float)(ux0 * sin(a) + uy0 * cos(a));
    }
    return B2T_OK;
}

extern "C" b2t_status b2t_fan_views(uint32_t n_angles, uint32_t n_dets, float src_origin,
                                    float origin_det, float det_width, const float *angles,
                                    b2t_view2d *out)
{
    clear_error();
    if (!angles || !out) return fail(B2T_ERR_INVALID_ARG, "b2t_fan_views: null pointer");
    // genFanProjections (src/GeometryUtil2D.cpp:81-104) with float locals
    const double fOriginSource = src_origin, fOriginDetector = origin_det, fDetSize = det_width;
    float fSrcX0 = 0.0f;
    float fSrcY0 = (float)-fOriginSource;
    float fDetUX0 = (float)fDetSize;
    float fDetUY0 = 0.0f;
    float fDetSX0 = n_dets * fDetUX0 / -2.0f;
    float fDetSY0 = (float)fOriginDetector;
    for (uint32_t i = 0; i < n_angles; ++i) {
        double a = angles[i];
        b2t_view2d &p = out[i];
        p.src[0] = (float)(fSrcX0 * cos(a) - fSrcY0 * sin(a));
        p.src[1] = (float)(fSrcX0 * sin(a) + fSrcY0 * cos(a));
        p.det_s[0] = (float)(fDetSX0 * cos(a) - fDetSY0 * sin(a));
        p.det_s[1] = (float)(fDetSX0 * sin(a) + fDetSY0 * cos(a));
        p.det_u[0] = (float)(fDetUX0 * cos(a) - fDetUY0 * sin(a));
        p.det_u[1] = (float)(fDetUX0 * sin(a) + fDetUY0 * cos(a));
    }
    return B2T_OK;
}

extern "C" b2t_status b2t_vec_views2d(uint32_t n_angles, uint32_t n_dets, const double *data,
                                      b2t_view2d *out)
{
    clear_error();
    if (!data || !out) return fail(B2T_ERR_INVALID_ARG, "b2t_vec_views2d: null pointer");
    for (uint32_t i = 0; i < n_angles; ++i) {
        const double *d = data + 6 * (size_t)i;
        b2t_view2d &p = out[i];
        p.src[0] = (float)d[0];
        p.src[1] = (float)d[1];
        p.det_u[0] = (float)d[4];
        p.det_u[1] = (float)d[5];
        p.det_s[0] = (float)(d[2] - 0.5 * n_dets * p.det_u[0]);
        p.det_s[1] = (float)(d[3] - 0.5 * n_dets * p.det_u[1]);
    }
    return B2T_OK;
}

extern "C" b2t_status b2t_normalize_views2d(const b2t_volgeom2d *vol, int32_t kind, uint32_t n,
                                            b2t_view2d *views, float *output_scale)
{
    clear_error();
    if (!vol || !views || !output_scale)
        return fail(B2T_ERR_INVALID_ARG, "b2t_normalize_views2d: null pointer");
    if (kind != B2T_GEOM_PAR2D && kind != B2T_GEOM_FAN2D)
        return fail(B2T_ERR_INVALID_ARG, "b2t_normalize_views2d: kind must be PAR2D or FAN2D");
    if (vol->cols == 0 || vol->rows == 0)
        return fail(B2T_ERR_INVALID_ARG, "b2t_normalize_views2d: empty volume");
    float lenX = vol->max_x - vol->min_x;
    float lenY = vol->max_y - vol->min_y;
    float pixX = lenX / (float)vol->cols;
    float pixY = lenY / (float)vol->rows;
    const float EPS = 0.00001f;
    if (std::abs(pixX - pixY) > EPS)
        return fail(B2T_ERR_UNSUPPORTED, "b2t_normalize_views2d: pixels must be square");
    float dx = -(vol->min_x + vol->max_x) / 2;
    float dy = -(vol->min_y + vol->max_y) / 2;
    float factor = 1.0f / pixX;
    for (uint32_t i = 0; i < n; ++i) {
        b2t_view2d &p = views[i];
        if (kind == B2T_GEOM_FAN2D) {
            p.src[0] = (float)(p.src[0] + (double)dx);
            p.src[1] = (float)(p.src[1] + (double)dy);
        }
        p.det_s[0] = (float)(p.det_s[0] + (double)dx);
        p.det_s[1] = (float)(p.det_s[1] + (double)dy);
        p.src[0] = (float)(p.src[0] * (double)factor);
        p.src[1] = (float)(p.src[1] * (double)factor);
        p.det_s[0] = (float)(p.det_s[0] * (double)factor);
        p.det_s[1] = (float)(p.det_s[1] * (double)factor);
        p.det_u[0] = (float)(p.det_u[0] * (double)factor);
        p.det_u[1] = (float)(p.det_u[1] * (double)factor);
    }
    *output_scale = 1.0f * pixX;
    return B2T_OK;
}
