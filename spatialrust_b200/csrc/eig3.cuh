// eig3.cuh -- smallest eigenpair of a symmetric 3x3 matrix, in FP32 or FP64.
//
// Eigenvalues: the closed-form trigonometric solution of the characteristic
// cubic (O. K. Smith, "Eigenvalues of a symmetric 3x3 matrix", CACM 4(4),
// 1961) -- the same method the reference uses in f32
// (crates/spatialrust-features/src/normal.rs:506-542).
// Eigenvector of the smallest eigenvalue: the longest cross product of two
// rows of (A - l0 I) (normal.rs:544-573).  When that product degenerates
// (l0 numerically repeated) a cyclic Jacobi iteration (Golub & Van Loan,
// Matrix Computations, sec. 8.5) is used instead -- the reference's own FP64
// fallback is also Jacobi (crates/spatialrust-math/src/eigen.rs:16-84).
#pragma once

namespace srcu {

struct Eig3 {
  double l0, l1, l2;  // ascending
  double v[3];        // unit eigenvector of l0
  bool jacobi;        // the Jacobi fallback was used
};

// Precision-dependent pieces of the solver (float: the fast path of the
// normal estimator; double: its refinement and the reference-precision path).
template <class T> struct EigTraits;
template <> struct EigTraits<double> {
  static constexpr double tiny = 1e-300, off_tol = 1e-34, cross_tol = 1e-12;
  __device__ static double sqrt_(double x) { return sqrt(x); }
  __device__ static double rsqrt_(double x) { return rsqrt(x); }
  __device__ static double acos_(double x) { return acos(x); }
  __device__ static double cos_(double x) { return cos(x); }
};
template <> struct EigTraits<float> {
  static constexpr float tiny = 1e-30f, off_tol = 1e-13f, cross_tol = 1e-6f;
  __device__ static float sqrt_(float x) { return sqrtf(x); }
  __device__ static float rsqrt_(float x) { return rsqrtf(x); }
  __device__ static float acos_(float x) { return acosf(x); }
  __device__ static float cos_(float x) { return cosf(x); }
};

template <class T>
__device__ __forceinline__ void sort3(T &a, T &b, T &c) {
  if (a > b) { T t = a; a = b; b = t; }
  if (b > c) { T t = b; b = c; c = t; }
  if (a > b) { T t = a; a = b; b = t; }
}

template <class T>
__device__ inline void jacobi_sym3(const T (&m)[3][3], Eig3 &r) {
  using Tr = EigTraits<T>;
  T a[3][3], v[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) a[i][j] = m[i][j];
  const T scale = fabs(a[0][0]) + fabs(a[1][1]) + fabs(a[2][2]) + Tr::tiny;
  for (int sweep = 0; sweep < 16; ++sweep) {
    const T off = a[0][1] * a[0][1] + a[0][2] * a[0][2] + a[1][2] * a[1][2];
    if (off <= Tr::off_tol * scale * scale) break;
#pragma unroll
    for (int pq = 0; pq < 3; ++pq) {
      const int p = pq == 2 ? 1 : 0;
      const int q = pq == 0 ? 1 : 2;
      const T apq = a[p][q];
      if (apq == T(0)) continue;
      const T theta = (a[q][q] - a[p][p]) / (T(2) * apq);
      const T t = (theta >= T(0) ? T(1) : T(-1)) / (fabs(theta) + Tr::sqrt_(T(1) + theta * theta));
      const T c = T(1) / Tr::sqrt_(T(1) + t * t);
      const T s = t * c;
      // A <- J^T A J with J the (p,q) rotation [c s; -s c]
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const T akp = a[k][p], akq = a[k][q];
        a[k][p] = c * akp - s * akq;
        a[k][q] = s * akp + c * akq;
      }
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const T apk = a[p][k], aqk = a[q][k];
        a[p][k] = c * apk - s * aqk;
        a[q][k] = s * apk + c * aqk;
      }
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const T vkp = v[k][p], vkq = v[k][q];
        v[k][p] = c * vkp - s * vkq;
        v[k][q] = s * vkp + c * vkq;
      }
    }
  }
  int imin = 0;
  if (a[1][1] < a[imin][imin]) imin = 1;
  if (a[2][2] < a[imin][imin]) imin = 2;
  T l[3] = {a[0][0], a[1][1], a[2][2]};
  r.v[0] = v[0][imin];
  r.v[1] = v[1][imin];
  r.v[2] = v[2][imin];
  sort3(l[0], l[1], l[2]);
  r.l0 = l[0];
  r.l1 = l[1];
  r.l2 = l[2];
  r.jacobi = true;
}

template <class T>
__device__ inline Eig3 smallest_eigenpair_t(T a00, T a11, T a22, T a01, T a02, T a12) {
  using Tr = EigTraits<T>;
  Eig3 r;
  r.jacobi = false;
  const T p1 = a01 * a01 + a02 * a02 + a12 * a12;
  const T q = (a00 + a11 + a22) / T(3);
  const T b00 = a00 - q, b11 = a11 - q, b22 = a22 - q;
  const T p2 = b00 * b00 + b11 * b11 + b22 * b22 + T(2) * p1;
  const T p = Tr::sqrt_(p2 / T(6));
  if (p1 == T(0) || p == T(0)) {
    T m[3][3] = {{a00, a01, a02}, {a01, a11, a12}, {a02, a12, a22}};
    jacobi_sym3(m, r);
    r.jacobi = p1 != T(0);  // a diagonal matrix is exact, not a fallback
    return r;
  }
  const T ip = T(1) / p;
  const T n00 = b00 * ip, n11 = b11 * ip, n22 = b22 * ip;
  const T n01 = a01 * ip, n02 = a02 * ip, n12 = a12 * ip;
  const T det = n00 * (n11 * n22 - n12 * n12) - n01 * (n01 * n22 - n12 * n02) +
                n02 * (n01 * n12 - n11 * n02);
  const T rr = fmin(T(1), fmax(T(-1), T(0.5) * det));
  const T phi = Tr::acos_(rr) / T(3);
  const T two_pi_3 = T(2.0943951023931954923);  // 2*pi/3
  T l2 = q + T(2) * p * Tr::cos_(phi);
  T l0 = q + T(2) * p * Tr::cos_(phi + two_pi_3);
  T l1 = T(3) * q - l0 - l2;
  sort3(l0, l1, l2);
  r.l0 = l0;
  r.l1 = l1;
  r.l2 = l2;
  // Rows of (A - l0 I); the eigenvector is orthogonal to all of them.
  const T r0[3] = {a00 - l0, a01, a02};
  const T r1[3] = {a01, a11 - l0, a12};
  const T r2[3] = {a02, a12, a22 - l0};
  T c[3][3];
  c[0][0] = r0[1] * r1[2] - r0[2] * r1[1];
  c[0][1] = r0[2] * r1[0] - r0[0] * r1[2];
  c[0][2] = r0[0] * r1[1] - r0[1] * r1[0];
  c[1][0] = r0[1] * r2[2] - r0[2] * r2[1];
  c[1][1] = r0[2] * r2[0] - r0[0] * r2[2];
  c[1][2] = r0[0] * r2[1] - r0[1] * r2[0];
  c[2][0] = r1[1] * r2[2] - r1[2] * r2[1];
  c[2][1] = r1[2] * r2[0] - r1[0] * r2[2];
  c[2][2] = r1[0] * r2[1] - r1[1] * r2[0];
  int best = 0;
  T bn = c[0][0] * c[0][0] + c[0][1] * c[0][1] + c[0][2] * c[0][2];
#pragma unroll
  for (int i = 1; i < 3; ++i) {
    const T nn = c[i][0] * c[i][0] + c[i][1] * c[i][1] + c[i][2] * c[i][2];
    if (nn > bn) {
      bn = nn;
      best = i;
    }
  }
  // The cross product's length is ~ (l1 - l0)(l2 - l0); when the gap to the
  // next eigenvalue is tiny against the spread the direction is dominated by
  // rounding, so use Jacobi.
  const T spread = l2 - l0;
  if (!(bn > Tr::cross_tol * spread * spread * spread * spread)) {
    T m[3][3] = {{a00, a01, a02}, {a01, a11, a12}, {a02, a12, a22}};
    jacobi_sym3(m, r);
    return r;
  }
  const T inv = Tr::rsqrt_(bn);
  r.v[0] = c[best][0] * inv;
  r.v[1] = c[best][1] * inv;
  r.v[2] = c[best][2] * inv;
  return r;
}

__device__ inline Eig3 smallest_eigenpair(double a00, double a11, double a22, double a01,
                                          double a02, double a12) {
  return smallest_eigenpair_t<double>(a00, a11, a22, a01, a02, a12);
}

}  // namespace srcu
