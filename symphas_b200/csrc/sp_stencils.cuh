/*
 * sp_stencils.cuh -- second- and fourth-order finite-difference stencils on an
 * accessor.
 *
 * Every point variant of SymPhas's 2nd-order stencils (sol/inc/stencilh2.h:
 * 2D :87-221, 3D :235-507), written with the summation order of the
 * reference so that, compiled without FMA contraction in FP64, a kernel gives
 * the same bits as the CPU solver.  The neighbour names follow the reference's
 * (sol/inc/stencil.h:975-1148): vx = +1 in x, vx_ = -1 in x, vx2y_ = (+2,-1) ...
 *
 * `a` is any accessor with a member template at<i,j,k>() returning the value at
 * offset (i,j,k) from the evaluated site; offsets are compile-time constants so
 * every shared-memory address folds to base + immediate.  Constants are cast to
 * the kernel's type T (K(x)), so FP32 kernels do no FP64 arithmetic.
 *
 * Quirks kept on purpose because the reference has them: lap_pts<3,19> reads vz
 * twice instead of vz + vz_ (stencilh2.h:273); gradlap_pts returns only the x
 * component (stencilh2.h:178-221, :417-507).
 */
#pragma once

namespace sp {
namespace st {

#define K(x) T(x)
#define P(i, j, k) a.template at<i, j, k>()
#define v0 P(0, 0, 0)
#define vx P(1, 0, 0)
#define vx_ P(-1, 0, 0)
#define vy P(0, 1, 0)
#define vy_ P(0, -1, 0)
#define vz P(0, 0, 1)
#define vz_ P(0, 0, -1)
#define vx2 P(2, 0, 0)
#define vx2_ P(-2, 0, 0)
#define vy2 P(0, 2, 0)
#define vy2_ P(0, -2, 0)
#define vz2 P(0, 0, 2)
#define vz2_ P(0, 0, -2)
#define vxy P(1, 1, 0)
#define vxy_ P(1, -1, 0)
#define vx_y P(-1, 1, 0)
#define vx_y_ P(-1, -1, 0)
#define vx2y P(2, 1, 0)
#define vx2y_ P(2, -1, 0)
#define vx2_y P(-2, 1, 0)
#define vx2_y_ P(-2, -1, 0)
#define vxy2 P(1, 2, 0)
#define vxy2_ P(1, -2, 0)
#define vx_y2 P(-1, 2, 0)
#define vx_y2_ P(-1, -2, 0)
#define vx2y2 P(2, 2, 0)
#define vx2y2_ P(2, -2, 0)
#define vx2_y2 P(-2, 2, 0)
#define vx2_y2_ P(-2, -2, 0)
#define vxz P(1, 0, 1)
#define vxz_ P(1, 0, -1)
#define vx_z P(-1, 0, 1)
#define vx_z_ P(-1, 0, -1)
#define vx2z P(2, 0, 1)
#define vx2z_ P(2, 0, -1)
#define vx2_z P(-2, 0, 1)
#define vx2_z_ P(-2, 0, -1)
#define vxz2 P(1, 0, 2)
#define vxz2_ P(1, 0, -2)
#define vx_z2 P(-1, 0, 2)
#define vx_z2_ P(-1, 0, -2)
#define vx2z2 P(2, 0, 2)
#define vx2z2_ P(2, 0, -2)
#define vx2_z2 P(-2, 0, 2)
#define vx2_z2_ P(-2, 0, -2)
#define vyz P(0, 1, 1)
#define vyz_ P(0, 1, -1)
#define vy_z P(0, -1, 1)
#define vy_z_ P(0, -1, -1)
#define vyz2 P(0, 1, 2)
#define vyz2_ P(0, 1, -2)
#define vy_z2 P(0, -1, 2)
#define vy_z2_ P(0, -1, -2)
#define vy2z P(0, 2, 1)
#define vy2z_ P(0, 2, -1)
#define vy2_z P(0, -2, 1)
#define vy2_z_ P(0, -2, -1)
#define vy2z2 P(0, 2, 2)
#define vy2z2_ P(0, 2, -2)
#define vy2_z2 P(0, -2, 2)
#define vy2_z2_ P(0, -2, -2)
#define vxyz P(1, 1, 1)
#define vxyz_ P(1, 1, -1)
#define vxy_z P(1, -1, 1)
#define vxy_z_ P(1, -1, -1)
#define vx_yz P(-1, 1, 1)
#define vx_yz_ P(-1, 1, -1)
#define vx_y_z P(-1, -1, 1)
#define vx_y_z_ P(-1, -1, -1)
#define vx2yz P(2, 1, 1)
#define vx2yz_ P(2, 1, -1)
#define vx2y_z P(2, -1, 1)
#define vx2y_z_ P(2, -1, -1)
#define vx2_yz P(-2, 1, 1)
#define vx2_yz_ P(-2, 1, -1)
#define vx2_y_z P(-2, -1, 1)
#define vx2_y_z_ P(-2, -1, -1)
#define vxy2z P(1, 2, 1)
#define vxy2z_ P(1, 2, -1)
#define vxy2_z P(1, -2, 1)
#define vxy2_z_ P(1, -2, -1)
#define vx_y2z P(-1, 2, 1)
#define vx_y2z_ P(-1, 2, -1)
#define vx_y2_z P(-1, -2, 1)
#define vx_y2_z_ P(-1, -2, -1)
#define vxyz2 P(1, 1, 2)
#define vxyz2_ P(1, 1, -2)
#define vxy_z2 P(1, -1, 2)
#define vxy_z2_ P(1, -1, -2)
#define vx_yz2 P(-1, 1, 2)
#define vx_yz2_ P(-1, 1, -2)
#define vx_y_z2 P(-1, -1, 2)
#define vx_y_z2_ P(-1, -1, -2)
#define vx2y2z2 P(2, 2, 2)
#define vx2y2z2_ P(2, 2, -2)
#define vx2y2_z2 P(2, -2, 2)
#define vx2y2_z2_ P(2, -2, -2)
#define vx2_y2z2 P(-2, 2, 2)
#define vx2_y2z2_ P(-2, 2, -2)
#define vx2_y2_z2 P(-2, -2, 2)
#define vx2_y2_z2_ P(-2, -2, -2)

#define vx3 P(3, 0, 0)
#define vx3_ P(-3, 0, 0)
#define vy3 P(0, 3, 0)
#define vy3_ P(0, -3, 0)
#define vx3y P(3, 1, 0)
#define vx3y_ P(3, -1, 0)
#define vx3_y P(-3, 1, 0)
#define vx3_y_ P(-3, -1, 0)
#define vxy3 P(1, 3, 0)
#define vxy3_ P(1, -3, 0)
#define vx_y3 P(-1, 3, 0)
#define vx_y3_ P(-1, -3, 0)
#define vx3y3 P(3, 3, 0)
#define vx3y3_ P(3, -3, 0)
#define vx3_y3 P(-3, 3, 0)
#define vx3_y3_ P(-3, -3, 0)

template <int DIM, int N> struct lap_pts;
template <> struct lap_pts<2, 5> {
  template <class T, class A>
  __device__ __forceinline__ static T apply(const A& a, T divh2) {
    return (vx_ + vx + vy + vy_ - K(4.) * v0) * divh2;
  }
};
template <> struct lap_pts<2, 9> {
  template <class T, class A>
  __device__ __forceinline__ static T apply(const A& a, T divh2) {
    return (vx_y + vxy_ + vxy + vx_y_ + K(4.) * vx + K(4.) * vy + K(4.) * vy_ + K(4.) * vx_ - K(20.) * v0) * divh2 * K(1.0 / 6);
  }
};
template <> struct lap_pts<3, 7> {
  template <class T, class A>
  __device__ __forceinline__ static T apply(const A& a, T divh2) {
    return (vx_ + vx + vy + vy_ + vz + vz_ - K(6.) * v0) * divh2;
  }
};
template <> struct lap_pts<3, 15> {
  template <class T, class A>
  __device__ __forceinline__ static T apply(const A& a, T divh2) {
    return (vx_y_z_ + vxy_z_ + vx_yz_ + vxyz_ + vx_y_z + vxy_z + vx_yz + vxyz + K(8.) * (vx_ + vx + vy + vy_ + vz + vz_ - K(7.) * v0)) * divh2 * K(1.0 / 12);
  }
};
template <> struct lap_pts<3, 19> {
  template <class T, class A>
  __device__ __forceinline__ static T apply(const A& a, T divh2) {
    return (vx_y_ + vxy_ + vx_y + vxy + vx_z_ + vxz_ + vx_z + vxz + vy_z_ + vyz_ + vy_z + vyz + K(2.) * (vx_ + vx + vy + vy_ + vz + vz) - K(24.) * v0) * divh2 * K(1.0 / 6);
  }
};
template <> struct lap_pts<3, 21> {
  template <class T, class A>
  __device__ __forceinline__ static T apply(const A& a, T divh2) {
    return (-(vx_y_z_ + vxy_z_ + vx_yz_ + vxyz_ + vx_y_z + vxy_z + vx_yz + vxyz) + K(4.) * (vx_y_ + vxy_ + vx_y + vxy + vx_z_ + vxz_ + vx_z + vxz + vy_z_ + vyz_ + vy_z + vyz) + K(-40.) * v0) * divh2 * K(1.0 / 12);
  }
};
template <> struct lap_pts<3, 27> {
  template <class T, class A>
  __device__ __forceinline__ static T apply(const A& a, T divh2) {
    return (vx_y_z_ + vxy_z_ + vx_yz_ + vxyz_ + vx_y_z + vxy_z + vx_yz + vxyz + K(3.) * (vx_y_ + vxy_ + vx_y + vxy + vx_z_ + vxz_ + vx_z + vxz + vy_z_ + vyz_ + vy_z + vyz) + K(14.) * (vx_ + vx + vy + vy_ + vz + vz_) - K(128.) * v0) * divh2 * K(1.0 / 30);
  }
};

template <int DIM, int N> struct bilap_pts;
template <> struct bilap_pts<2, 13> {
  template <class T, class A>
  __device__ __forceinline__ static T apply(const A& a, T divh4) {
    return (vy2_ + vy2 + vx2_ + vx2 + K(2.) * (vx_y_ + vxy_ + vx_y + vxy) - K(8.) * (vx_ + vx + vy_ + vy) + K(20.) * v0) * divh4;
  }
};
template <> struct bilap_pts<2, 17> {
  template <class T, class A>
  __device__ __forceinline__ static T apply(const A& a, T divh4) {
    return ((vx2y2 + vx2_y2 + vx2y2_ + vx2_y2_) + K(10.) * (vx2 + vx2_ + vy2 + vy2_) + K(8.) * (vxy + vx_y + vxy_ + vx_y_) - K(64.) * (vx + vx_ + vy + vy_) + K(180.) * v0) * divh4 * K(1.0 / 12);
  }
};
template <> struct bilap_pts<2, 21> {
  template <class T, class A>
  __device__ __forceinline__ static T apply(const A& a, T divh4) {
    return ((vx2y + vx2_y + vx2y_ + vx2_y_ + vxy2 + vx_y2 + vxy2_ + vx_y2_) + (vx2 + vx2_ + vy2 + vy2_) - K(2.) * (vxy + vx_y + vxy_ + vx_y_) - K(10.) * (vx + vx_ + vy + vy_) + K(36.) * v0) * divh4 * K(1.0 / 12);
  }
};
template <> struct bilap_pts<3, 21> {
  template <class T, class A>
  __device__ __forceinline__ static T apply(const A& a, T divh4) {
    return ((vx2y2 + vx2_y2 + vx2y2_ + vx2_y2_ + vx2z2_ + vx2_z2_ + vx2z2 + vx2_z2 + vy2z2_ + vy2z2 + vy2_z2_ + vy2_z2) - K(4.) * (vxyz + vx_yz + vxy_z + vx_y_z + vxyz_ + vx_yz_ + vxy_z_ + vx_y_z_) + K(20.) * v0) * divh4 * K(1.0 / 4);
  }
};
template <> struct bilap_pts<3, 25> {
  template <class T, class A>
  __device__ __forceinline__ static T apply(const A& a, T divh4) {
    return (K(2.) * (vxy + vx_y + vxy_ + vx_y_ + vxz_ + vx_z_ + vxz + vx_z + vyz_ + vyz + vy_z_ + vy_z) + (vx2 + vx2_ + vy2 + vy2_ + vz2 + vz2_) - K(12.) * (vx + vx_ + vy + vy_ + vz + vz_) + K(42.) * v0) * divh4;
  }
};
template <> struct bilap_pts<3, 41> {
  template <class T, class A>
  __device__ __forceinline__ static T apply(const A& a, T divh4) {
    return ((vx2y2z2 + vx2_y2z2 + vx2y2_z2 + vx2_y2_z2 + vx2y2z2_ + vx2_y2z2_ + vx2y2_z2_ + vx2_y2_z2_) - K(40.) * (vxyz + vx_yz + vxy_z + vx_y_z + vxyz_ + vx_yz_ + vxy_z_ + vx_y_z_) + K(96.) * (vxy + vx_y + vxy_ + vx_y_ + vxz_ + vx_z_ + vxz + vx_z + vyz_ + vyz + vy_z_ + vy_z) + K(20.) * (vx2 + vx2_ + vy2 + vy2_ + vz2 + vz2_) - K(320.) * (vx + vx_ + vy + vy_ + vz + vz_) + K(960.) * v0) * divh4 * K(1.0 / 24);
  }
};
template <> struct bilap_pts<3, 52> {
  template <class T, class A>
  __device__ __forceinline__ static T apply(const A& a, T divh4) {
    return (-(vx2y2z2 + vx2_y2z2 + vx2y2_z2 + vx2_y2_z2 + vx2y2z2_ + vx2_y2z2_ + vx2y2_z2_ + vx2_y2_z2_) + K(10.) * (vxyz2 + vx_yz2 + vxy_z2 + vx_y_z2 + vxyz2_ + vx_yz2_ + vxy_z2_ + vx_y_z2_ + vxy2z + vx_y2z + vxy2_z + vx_y2_z + vxy2z_ + vx_y2z_ + vxy2_z_ + vx_y2_z_ + vx2yz + vx2_yz + vx2y_z + vx2_y_z + vx2yz_ + vx2_yz_ + vx2y_z_ + vx2_y_z_) - K(20.) * (vxyz + vx_yz + vxy_z + vx_y_z + vxyz_ + vx_yz_ + vxy_z_ + vx_y_z_) - K(36.) * (vxy + vx_y + vxy_ + vx_y_ + vxz_ + vx_z_ + vxz + vx_z + vyz_ + vyz + vy_z_ + vy_z) + K(360.) * v0) * divh4 * K(1.0 / 36);
  }
};
template <> struct bilap_pts<3, 57> {
  template <class T, class A>
  __device__ __forceinline__ static T apply(const A& a, T divh4) {
    return ((vyz2 + vy_z2 + vyz2_ + vy_z2_ + vy2z + vy2_z + vy2z_ + vy2_z_ + vx2z + vx2_z + vx2z_ + vx2_z_ + vxz2 + vx_z2 + vxz2_ + vx_z2_ + vxy2 + vx_y2 + vxy2_ + vx_y2_ + vx2y + vx2_y + vx2y_ + vx2_y_) + K(3.) * (vxyz + vx_yz + vxy_z + vx_y_z + vxyz_ + vx_yz_ + vxy_z_ + vx_y_z_) - K(8.) * (vxy + vx_y + vxy_ + vx_y_ + vxz_ + vx_z_ + vxz + vx_z + vyz_ + vyz + vy_z_ + vy_z) - (vx2 + vx2_ + vy2 + vy2_ + vz2 + vz2_) + K(4.) * (vx + vx_ + vy + vy_ + vz + vz_) + K(30.) * v0) * divh4 * K(1.0 / 3);
  }
};

template <int DIM, int N> struct gradlap_pts;
template <> struct gradlap_pts<2, 6> {
  template <class T, class A>
  __device__ __forceinline__ static T apply(const A& a, T divh3) {
    return ((vx2y - vx2_y + vx2y_ - vx2_y_) - K(4.) * (vx - vx_)) * divh3 * K(1.0 / 4);
  }
};
template <> struct gradlap_pts<2, 8> {
  template <class T, class A>
  __device__ __forceinline__ static T apply(const A& a, T divh3) {
    return ((vx2 - vx2_) + (vxy - vx_y + vxy_ - vx_y_) - K(4.) * (vx - vx_)) * divh3 * K(1.0 / 2);
  }
};
template <> struct gradlap_pts<2, 12> {
  template <class T, class A>
  __device__ __forceinline__ static T apply(const A& a, T divh3) {
    return ((vx2y2 - vx2_y2 + vx2y2_ - vx2_y2_) + K(10.) * (vx2 - vx2_) + K(4.) * (vxy - vx_y + vxy_ - vx_y_) - K(32.) * (vx - vx_)) * divh3 * K(1.0 / 24);
  }
};
template <> struct gradlap_pts<2, 16> {
  template <class T, class A>
  __device__ __forceinline__ static T apply(const A& a, T divh3) {
    return (K(2.) * (vx2y - vx2_y + vx2y_ - vx2_y_) + K(2.) * (vx2 - vx2_) + (vxy2 - vx_y2 + vxy2_ - vx_y2_) - K(2.) * (vxy - vx_y + vxy_ - vx_y_) - K(10.) * (vx - vx_)) * divh3 * K(1.0 / 12);
  }
};
template <> struct gradlap_pts<3, 10> {
  template <class T, class A>
  __device__ __forceinline__ static T apply(const A& a, T divh3) {
    return ((vx2yz - vx2_yz + vx2y_z - vx2_y_z + vx2yz_ - vx2_yz_ + vx2y_z_ - vx2_y_z_) - K(8.) * (vx - vx_)) * divh3 * K(1.0 / 8);
  }
};
template <> struct gradlap_pts<3, 12> {
  template <class T, class A>
  __device__ __forceinline__ static T apply(const A& a, T divh3) {
    return ((vx2 - vx2_) + (vxy - vx_y + vxy_ - vx_y_ + vxz_ - vx_z_ + vxz - vx_z) - K(6.) * (vx - vx_)) * divh3 * K(1.0 / 2);
  }
};
template <> struct gradlap_pts<3, 28> {
  template <class T, class A>
  __device__ __forceinline__ static T apply(const A& a, T divh3) {
    return ((vx2y2 - vx2_y2 + vx2y2_ - vx2_y2_ + vx2z2_ - vx2_z2_ + vx2z2 - vx2_z2) + K(8.) * (vx2 - vx2_) + K(6.) * (vxyz - vx_yz + vxy_z - vx_y_z + vxyz_ - vx_yz_ + vxy_z_ - vx_y_z_) - K(8.) * (vxy - vx_y + vxy_ - vx_y_ + vxz_ - vx_z_ + vxz - vx_z) - K(16.) * (vx - vx_)) * divh3 * K(1.0 / 24);
  }
};
template <> struct gradlap_pts<3, 36> {
  template <class T, class A>
  __device__ __forceinline__ static T apply(const A& a, T divh3) {
    return (K(2.) * (vx2z - vx2_z + vx2z_ - vx2_z_ + vx2y - vx2_y + vx2y_ - vx2_y_) - K(2.) * (vx2 - vx2_) + (vxz2 - vx_z2 + vxz2_ - vx_z2_ + vxy2 - vx_y2 + vxy2_ - vx_y2_) + K(3.) * (vxyz - vx_yz + vxy_z - vx_y_z + vxyz_ - vx_yz_ + vxy_z_ - vx_y_z_) - K(8.) * (vxy - vx_y + vxy_ - vx_y_ + vxz_ - vx_z_ + vxz - vx_z) + K(4.) * (vx - vx_)) * divh3 * K(1.0 / 12);
  }
};
template <> struct gradlap_pts<3, 40> {
  template <class T, class A>
  __device__ __forceinline__ static T apply(const A& a, T divh3) {
    return (K(16.) * (vx2z - vx2_z + vx2z_ - vx2_z_ + vx2y - vx2_y + vx2y_ - vx2_y_) - K(16.) * (vx2 - vx2_) + K(3.) * (vxy2z - vx_y2z + vxy2_z - vx_y2_z + vxy2z_ - vx_y2z_ + vxy2_z_ - vx_y2_z_ + vxyz2 - vx_yz2 + vxy_z2 - vx_y_z2 + vxyz2_ - vx_yz2_ + vxy_z2_ - vx_y_z2_) + K(2.) * (vxz2 - vx_z2 + vxz2_ - vx_z2_ + vxy2 - vx_y2 + vxy2_ - vx_y2_) - K(22.) * (vxy - vx_y + vxy_ - vx_y_ + vxz_ - vx_z_ + vxz - vx_z) - K(40.) * (vx - vx_)) * divh3 * K(1.0 / 96);
  }
};

// ---------------------------------------------------------------------------
// 4th-order 2D stencils (Stencil2d4h, sol/inc/stencilh4.h): every point set of
// the reference, in its summation order.  The `s` argument is the scale
// factor the reference passes: Stencil2d4h gives all three operators divh3
// (sol/inc/stencilincludes.h:446, :453, :460), so the Laplacian and the
// bilaplacian scale correctly only for h = 1; that behaviour is kept.
// ---------------------------------------------------------------------------
template <int N> struct lap4_pts;
template <> struct lap4_pts<9> {  // stencilh4.h:44-53
  template <class T, class A>
  __device__ __forceinline__ static T apply(const A& a, T s) {
    return (-vx2_ - vx2 - vy2 - vy2_ + K(16.) * (vx_ + vx + vy + vy_) - K(60.) * v0) * s * K(1.0 / 12);
  }
};
template <> struct lap4_pts<17> {  // stencilh4.h:55-67
  template <class T, class A>
  __device__ __forceinline__ static T apply(const A& a, T s) {
    return (-(vx2y2 + vx2_y2 + vx2y2_ + vx2_y2_) - K(8.) * (vx2 + vx2_ + vy2 + vy2_) +
            K(16.) * (vxy + vx_y + vxy_ + vx_y_) + K(128.) * (vx + vx_ + vy + vy_) - K(540.) * v0) *
           s * K(1.0 / 120);
  }
};
template <> struct lap4_pts<21> {  // stencilh4.h:69-82
  template <class T, class A>
  __device__ __forceinline__ static T apply(const A& a, T s) {
    return (-K(2.) * (vx2y + vx2_y + vx2y_ + vx2_y_ + vxy2 + vx_y2 + vxy2_ + vx_y2_) -
            (vx2 + vx2_ + vy2 + vy2_) + K(16.) * (vxy + vx_y + vxy_ + vx_y_) +
            K(52.) * (vx + vx_ + vy + vy_) - K(252.) * v0) *
           s * K(1.0 / 60);
  }
};
template <int N> struct bilap4_pts;
template <> struct bilap4_pts<21> {  // stencilh4.h:85-98
  template <class T, class A>
  __device__ __forceinline__ static T apply(const A& a, T s) {
    return (-K(4.) * (vx3 + vx3_ + vy3 + vy3_) - (vx2y2 + vx2_y2 + vx2y2_ + vx2_y2_) +
            K(50.) * (vx2 + vx2_ + vy2 + vy2_) + K(64.) * (vxy + vx_y + vxy_ + vx_y_) -
            K(284.) * (vx + vx_ + vy + vy_) + K(700.) * v0) *
           s * K(1.0 / 24);
  }
};
template <> struct bilap4_pts<25> {  // stencilh4.h:100-113
  template <class T, class A>
  __device__ __forceinline__ static T apply(const A& a, T s) {
    return (-(vx3 + vx3_ + vy3 + vy3_) -
            (vx2y + vx2_y + vx2y_ + vx2_y_ + vxy2 + vx_y2 + vxy2_ + vx_y2_) +
            K(14.) * (vx2 + vx2_ + vy2 + vy2_) + K(20.) * (vxy + vx_y + vxy_ + vx_y_) -
            K(77.) * (vx + vx_ + vy + vy_) + K(184.) * v0) *
           s * K(1.0 / 6);
  }
};
template <> struct bilap4_pts<33> {  // stencilh4.h:115-131
  template <class T, class A>
  __device__ __forceinline__ static T apply(const A& a, T s) {
    return (-K(17.) * (vx3y3 + vx3_y3 + vx3y3_ + vx3_y3_) - K(236.) * (vx3 + vx3_ + vy3 + vy3_) +
            K(351.) * (vx2y2 + vx2_y2 + vx2y2_ + vx2_y2_) -
            K(756.) * (vx2y + vx2_y + vx2y_ + vx2_y_ + vxy2 + vx_y2 + vxy2_ + vx_y2_) +
            K(4050.) * (vx2 + vx2_ + vy2 + vy2_) + K(5049.) * (vxy + vx_y + vxy_ + vx_y_) -
            K(19116.) * (vx + vx_ + vy + vy_) + K(45724.) * v0) *
           s * K(1.0 / 1620);
  }
};
template <> struct bilap4_pts<37> {  // stencilh4.h:133-148
  template <class T, class A>
  __device__ __forceinline__ static T apply(const A& a, T s) {
    return (-K(17.) * (vx3y + vx3_y + vx3y_ + vx3_y_ + vxy3 + vx_y3 + vxy3_ + vx_y3_) +
            K(4.) * (vx3 + vx3_ + vy3 + vy3_) - K(29.) * (vx2y2 + vx2_y2 + vx2y2_ + vx2_y2_) +
            K(188.) * (vx2y + vx2_y + vx2y_ + vx2_y_ + vxy2 + vx_y2 + vxy2_ + vx_y2_) +
            K(42.) * (vx2 + vx2_ + vy2 + vy2_) - K(374.) * (vxy + vx_y + vxy_ + vx_y_) -
            K(764.) * (vx + vx_ + vy + vy_) + K(3116.) * v0) *
           s * K(1.0 / 180);
  }
};
// gradlaplacians: the x component, as the reference returns
template <int N> struct gradlap4_pts;
template <> struct gradlap4_pts<14> {  // stencilh4.h:150-163
  template <class T, class A>
  __device__ __forceinline__ static T apply(const A& a, T s) {
    return (-K(6.) * (vx3 - vx3_) - (vx2y2 - vx2_y2 + vx2y2_ - vx2_y2_) + K(50.) * (vx2 - vx2_) +
            K(32.) * (vxy - vx_y + vxy_ - vx_y_) - K(142.) * (vx - vx_)) *
           s * K(1.0 / 48);
  }
};
template <> struct gradlap4_pts<18> {  // stencilh4.h:165-179
  template <class T, class A>
  __device__ __forceinline__ static T apply(const A& a, T s) {
    return (-K(3.) * (vx3) - K(2.) * (vx2y - vx2_y + vx2y_ - vx2_y_) + K(28.) * (vx2) -
            (vxy2 - vx_y2 + vxy2_ - vx_y2_) + K(20.) * (vxy - vx_y + vxy_ - vx_y_) - K(77.) * (vx)) *
           s * K(1.0 / 24);
  }
};
template <> struct gradlap4_pts<26> {  // stencilh4.h:181-197: divides by 2160 s
  template <class T, class A>
  __device__ __forceinline__ static T apply(const A& a, T s) {
    return (-K(17.) * (vx3y3 - vx3_y3 + vx3y3_ - vx3_y3_) - K(236.) * (vx3) +
            K(234.) * (vx2y2 - vx2_y2 + vx2y2_ - vx2_y2_) - K(504.) * (vx2y - vx2_y + vx2y_ - vx2_y_) +
            K(2700.) * (vx2) - K(252.) * (vxy2 - vx_y2 + vxy2_ - vx_y2_) +
            K(1683.) * (vxy - vx_y + vxy_ - vx_y_) - K(6372.) * (vx)) /
           (K(2160.) * s);
  }
};
template <> struct gradlap4_pts<30> {  // stencilh4.h:199-216
  template <class T, class A>
  __device__ __forceinline__ static T apply(const A& a, T s) {
    return (-K(51.) * (vx3y - vx3_y + vx3y_ - vx3_y_) + K(12.) * (vx3) -
            K(58.) * (vx2y2 - vx2_y2 + vx2y2_ - vx2_y2_) + K(376.) * (vx2y - vx2_y + vx2y_ - vx2_y_) +
            K(84.) * (vx2) - K(17.) * (vxy3 - vx_y3 + vxy3_ - vx_y3_) +
            K(188.) * (vxy2 - vx_y2 + vxy2_ - vx_y2_) - K(374.) * (vxy - vx_y + vxy_ - vx_y_) -
            K(764.) * (vx)) *
           s * K(1.0 / 720);
  }
};

#undef vx3
#undef vx3_
#undef vy3
#undef vy3_
#undef vx3y
#undef vx3y_
#undef vx3_y
#undef vx3_y_
#undef vxy3
#undef vxy3_
#undef vx_y3
#undef vx_y3_
#undef vx3y3
#undef vx3y3_
#undef vx3_y3
#undef vx3_y3_

#undef P
#undef v0
#undef vx
#undef vx_
#undef vy
#undef vy_
#undef vz
#undef vz_
#undef vx2
#undef vx2_
#undef vy2
#undef vy2_
#undef vz2
#undef vz2_
#undef vxy
#undef vxy_
#undef vx_y
#undef vx_y_
#undef vx2y
#undef vx2y_
#undef vx2_y
#undef vx2_y_
#undef vxy2
#undef vxy2_
#undef vx_y2
#undef vx_y2_
#undef vx2y2
#undef vx2y2_
#undef vx2_y2
#undef vx2_y2_
#undef vxz
#undef vxz_
#undef vx_z
#undef vx_z_
#undef vx2z
#undef vx2z_
#undef vx2_z
#undef vx2_z_
#undef vxz2
#undef vxz2_
#undef vx_z2
#undef vx_z2_
#undef vx2z2
#undef vx2z2_
#undef vx2_z2
#undef vx2_z2_
#undef vyz
#undef vyz_
#undef vy_z
#undef vy_z_
#undef vyz2
#undef vyz2_
#undef vy_z2
#undef vy_z2_
#undef vy2z
#undef vy2z_
#undef vy2_z
#undef vy2_z_
#undef vy2z2
#undef vy2z2_
#undef vy2_z2
#undef vy2_z2_
#undef vxyz
#undef vxyz_
#undef vxy_z
#undef vxy_z_
#undef vx_yz
#undef vx_yz_
#undef vx_y_z
#undef vx_y_z_
#undef vx2yz
#undef vx2yz_
#undef vx2y_z
#undef vx2y_z_
#undef vx2_yz
#undef vx2_yz_
#undef vx2_y_z
#undef vx2_y_z_
#undef vxy2z
#undef vxy2z_
#undef vxy2_z
#undef vxy2_z_
#undef vx_y2z
#undef vx_y2z_
#undef vx_y2_z
#undef vx_y2_z_
#undef vxyz2
#undef vxyz2_
#undef vxy_z2
#undef vxy_z2_
#undef vx_yz2
#undef vx_yz2_
#undef vx_y_z2
#undef vx_y_z2_
#undef vx2y2z2
#undef vx2y2z2_
#undef vx2y2_z2
#undef vx2y2_z2_
#undef vx2_y2z2
#undef vx2_y2z2_
#undef vx2_y2_z2
#undef vx2_y2_z2_

#undef K

// reach (Chebyshev radius) of each operator's point set
template <int DIM, int N> struct lap_reach { static constexpr int value = 1; };
template <int DIM, int N> struct bilap_reach { static constexpr int value = 2; };
template <int DIM, int N> struct gradlap_reach { static constexpr int value = 2; };

}  // namespace st
}  // namespace sp
