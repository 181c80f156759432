// host_math.hpp -- host-side small-matrix arithmetic for the NICP library.
//
// The projector matrices handed to the kernels are computed here in float,
// in the reference's order of operations (pinholepointprojector.cpp:16-31):
// every fixed-size product accumulates sequentially over the inner index
// with no fused multiply-add (this file is compiled with
// -ffp-contract=off), the 3x3 camera inverse is the adjugate times the
// reciprocal determinant, and the isometry inverse is [R^T, -R^T t].
#pragma once
#include <cmath>
#include <cstring>

#include "nicp_gpu.h"

namespace nicp {

struct HM4 {
  float a[16];
  float &operator()(int r, int c) { return a[r * 4 + c]; }
  float operator()(int r, int c) const { return a[r * 4 + c]; }
  static HM4 identity() {
    HM4 m;
    for (int i = 0; i < 16; i++) m.a[i] = (i % 5 == 0) ? 1.0f : 0.0f;
    return m;
  }
  static HM4 from(const float *p) {
    if (!p) return identity();
    HM4 m;
    std::memcpy(m.a, p, sizeof(m.a));
    m.a[12] = 0.0f; m.a[13] = 0.0f; m.a[14] = 0.0f; m.a[15] = 1.0f;
    return m;
  }
};

inline HM4 hm_mul(const HM4 &A, const HM4 &B) {
  HM4 C;
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) {
      float s = A(i, 0) * B(0, j);
      s = s + A(i, 1) * B(1, j);
      s = s + A(i, 2) * B(2, j);
      s = s + A(i, 3) * B(3, j);
      C(i, j) = s;
    }
  return C;
}

inline HM4 hm_iso_inverse(const HM4 &T) {
  HM4 r = HM4::identity();
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) r(i, j) = T(j, i);
  for (int i = 0; i < 3; i++) {
    float s = r(i, 0) * T(0, 3);
    s = s + r(i, 1) * T(1, 3);
    s = s + r(i, 2) * T(2, 3);
    r(i, 3) = -s;
  }
  return r;
}

inline void hm_inv3(const float m[9], float out[9]) {
  float c00 = m[4] * m[8] - m[5] * m[7];
  float c01 = m[5] * m[6] - m[3] * m[8];
  float c02 = m[3] * m[7] - m[4] * m[6];
  float det = m[0] * c00;
  det = det + m[1] * c01;
  det = det + m[2] * c02;
  float id = 1.0f / det;
  out[0] = c00 * id;
  out[3] = c01 * id;
  out[6] = c02 * id;
  out[1] = (m[2] * m[7] - m[1] * m[8]) * id;
  out[4] = (m[0] * m[8] - m[2] * m[6]) * id;
  out[7] = (m[1] * m[6] - m[0] * m[7]) * id;
  out[2] = (m[1] * m[5] - m[2] * m[4]) * id;
  out[5] = (m[2] * m[3] - m[0] * m[5]) * id;
  out[8] = (m[0] * m[4] - m[1] * m[3]) * id;
}

// Effective camera matrix: rows 0..1 of the original times the scaling
// factor (pinholepointprojector.cpp:150-155).
inline void cam_K(const nicp_camera &c, float K[9]) {
  float K0[9] = {c.fx, 0.0f, c.cx, 0.0f, c.fy, c.cy, 0.0f, 0.0f, 1.0f};
  for (int i = 0; i < 9; i++) K[i] = (i < 6) ? K0[i] * c.scaling : K0[i];
}
inline int cam_rows(const nicp_camera &c) { return (int)((float)c.rows * c.scaling); }
inline int cam_cols(const nicp_camera &c) { return (int)((float)c.cols * c.scaling); }

// _updateMatrices(): KRt = [K R(T^-1) | K t(T^-1)], iKRt = [R(T) K^-1 | t(T)].
inline void projector_matrices(const nicp_camera &c, const HM4 &transform, HM4 &KRt, HM4 &iKRt) {
  float K[9], iK[9];
  cam_K(c, K);
  hm_inv3(K, iK);
  HM4 t = hm_iso_inverse(transform);
  KRt = HM4::identity();
  iKRt = HM4::identity();
  for (int i = 0; i < 3; i++) {
    for (int j = 0; j < 3; j++) {
      float s = K[i * 3 + 0] * t(0, j);
      s = s + K[i * 3 + 1] * t(1, j);
      s = s + K[i * 3 + 2] * t(2, j);
      KRt(i, j) = s;
      float u = transform(i, 0) * iK[0 * 3 + j];
      u = u + transform(i, 1) * iK[1 * 3 + j];
      u = u + transform(i, 2) * iK[2 * 3 + j];
      iKRt(i, j) = u;
    }
    float s = K[i * 3 + 0] * t(0, 3);
    s = s + K[i * 3 + 1] * t(1, 3);
    s = s + K[i * 3 + 2] * t(2, 3);
    KRt(i, 3) = s;
    iKRt(i, 3) = transform(i, 3);
  }
}

}  // namespace nicp
