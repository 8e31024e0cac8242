// host_inst.cpp - instance transforms on the host: composition from translate / axis-angle / scale with per-frame
// velocities, and the FP64 inverse that the two-level traversal uses to bring rays into object space.
#include "cwp_b200.h"
#include "runtime.h"
#include <cmath>

using namespace cwpb;

// Inverse of the affine 3x4 map m (rows m0 m1 m2 t): adjugate over determinant in double, translation -(A^-1 t),
// rounded to float once (scene/instances.cpp:64-79). A singular matrix gives a zero inverse and det sign +1.
extern "C" int cwp_xform_invert(const float m[12], float inv[12], float* det_sign) {
    CWPB_CHECK(m && inv, CWP_ERR_INVALID, "NULL matrix");
    const double a00 = m[0], a01 = m[1], a02 = m[2], a10 = m[4], a11 = m[5], a12 = m[6], a20 = m[8], a21 = m[9], a22 = m[10];
    // cofactors of the first row give the determinant; the adjugate is the transposed cofactor matrix
    const double c00 = a11 * a22 - a12 * a21, c01 = a12 * a20 - a10 * a22, c02 = a10 * a21 - a11 * a20;
    const double det = a00 * c00 + a01 * c01 + a02 * c02;
    const double r = det != 0.0 ? 1.0 / det : 0.0;
    double b[3][3];
    b[0][0] = c00 * r;                        b[0][1] = (a02 * a21 - a01 * a22) * r; b[0][2] = (a01 * a12 - a02 * a11) * r;
    b[1][0] = c01 * r;                        b[1][1] = (a00 * a22 - a02 * a20) * r; b[1][2] = (a02 * a10 - a00 * a12) * r;
    b[2][0] = c02 * r;                        b[2][1] = (a01 * a20 - a00 * a21) * r; b[2][2] = (a00 * a11 - a01 * a10) * r;
    const double t[3] = { m[3], m[7], m[11] };
    for (int i = 0; i < 3; i++) {
        for (int j = 0; j < 3; j++) inv[4 * i + j] = (float)b[i][j];
        inv[4 * i + 3] = (float)(-(b[i][0] * t[0] + b[i][1] * t[1] + b[i][2] * t[2]));
    }
    if (det_sign) *det_sign = det < 0.0 ? -1.f : 1.f;
    return CWP_OK;
}

// m = T(translate + f v_t) R(axis, angle + f v_a) S(scale + f v_s), composed in double and rounded once
// (scene/instances.cpp:48-62); a zero axis means +z.
extern "C" int cwp_xform_animate(const cwp_instance_desc* d, int32_t frame, float m[12]) {
    CWPB_CHECK(d && m, CWP_ERR_INVALID, "NULL argument");
    const double f = frame;
    double t[3], s[3];
    for (int i = 0; i < 3; i++) { t[i] = d->translate[i] + f * d->translate_per_frame[i]; s[i] = d->scale[i] + f * d->scale_per_frame[i]; }
    const double ang = (d->angle_deg + f * d->angle_deg_per_frame) * (3.14159265358979323846 / 180.0);
    double x = d->axis[0], y = d->axis[1], z = d->axis[2];
    const double len = std::sqrt(x * x + y * y + z * z);
    if (len > 0.0) { x /= len; y /= len; z /= len; } else { x = 0.0; y = 0.0; z = 1.0; }
    const double c = std::cos(ang), sn = std::sin(ang), k = 1.0 - c;
    // Rodrigues: R = c I + sin [axis]x + (1 - c) axis axis^T
    const double R[3][3] = { { c + x * x * k, x * y * k - z * sn, x * z * k + y * sn },
                             { y * x * k + z * sn, c + y * y * k, y * z * k - x * sn },
                             { z * x * k - y * sn, z * y * k + x * sn, c + z * z * k } };
    for (int i = 0; i < 3; i++) {
        for (int j = 0; j < 3; j++) m[4 * i + j] = (float)(R[i][j] * s[j]);
        m[4 * i + 3] = (float)t[i];
    }
    return CWP_OK;
}

extern "C" int cwp_instance_from_xform(const float m[12], int32_t mesh, cwp_instance* out) {
    CWPB_CHECK(m && out, CWP_ERR_INVALID, "NULL argument");
    CWPB_CHECK(mesh >= 0, CWP_ERR_INVALID, "negative mesh index %d", mesh);
    for (int i = 0; i < 12; i++) out->fwd[i] = m[i];
    if (int rc = cwp_xform_invert(m, out->inv, &out->det_sign)) return rc;
    out->root = -1; out->mesh = mesh; out->pad = 0;
    return CWP_OK;
}
