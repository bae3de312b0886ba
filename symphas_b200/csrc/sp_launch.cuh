/*
 * sp_launch.cuh -- turns a model factory into a registered kernel entry.
 */
#pragma once

#include <utility>

#include "sp_ch.cuh"
#include "sp_chrow.cuh"
#include "sp_row.cuh"
#include "sp_kernels.cuh"
#include "sp_models.cuh"
#include "sp_tb2.cuh"
#include "sp_registry.h"

namespace sp {

// Launches a step kernel with programmatic stream serialization: its grid may
// start while the previous kernel in the stream drains.  Every step kernel
// calls pdl_enter() before its first global access.
template <class... KArgs, class... Args>
cudaError_t launch_step_kernel(void (*kern)(KArgs...), dim3 grid, int nt, size_t smem,
                               cudaStream_t s, Args&&... args) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = grid;
  cfg.blockDim = dim3(nt);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...);
}

template <class MF>
using model_of = decltype(MF{}());

template <class MF, class T, int LP, int GP, int BP, class TC, bool EXACT>
struct Entry3 {
  using M = model_of<MF>;
  using K = Fd3<M, T, LP, GP, BP, TC, EXACT>;
  static cudaError_t launch(const void* prm, dim3 grid, cudaStream_t s) {
    auto kern = k_fd3d<M, T, LP, GP, BP, TC, EXACT>;
    static cudaError_t attr = cudaFuncSetAttribute(
        kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(K::SMEM));
    if (attr != cudaSuccess) return attr;
    const M m = MF{}();
    return launch_step_kernel(kern, grid, K::NT, K::SMEM, s,
                              *static_cast<const StepParams<T>*>(prm), m);
  }
  static int occupancy() {
    auto kern = k_fd3d<M, T, LP, GP, BP, TC, EXACT>;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(K::SMEM));
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, K::NT, K::SMEM) != cudaSuccess)
      return 1;
    return n > 0 ? n : 1;
  }
  static KernelInfo info() {
    return KernelInfo{K::NF, K::NS,     K::R,    K::HXA,  K::TX,      K::TY,
                      K::SPT, K::PD, K::NT, K::SMEM, &launch, &occupancy};
  }
};

// the conserved-pattern kernel (sp_ch.cuh) as a tile variant of a fused key
template <class MF, class T, class TC>
struct EntryCh3 {
  using M = model_of<MF>;
  using K = Ch3<M, T, TC>;
  static cudaError_t launch(const void* prm, dim3 grid, cudaStream_t s) {
    auto kern = k_ch3d<M, T, TC>;
    static cudaError_t attr = cudaFuncSetAttribute(
        kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(K::SMEM));
    if (attr != cudaSuccess) return attr;
    const M m = MF{}();
    return launch_step_kernel(kern, grid, K::NT, K::SMEM, s,
                              *static_cast<const StepParams<T>*>(prm), m);
  }
  static int occupancy() {
    auto kern = k_ch3d<M, T, TC>;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(K::SMEM));
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, K::NT, K::SMEM) != cudaSuccess)
      return 1;
    return n > 0 ? n : 1;
  }
  static KernelInfo info() {
    return KernelInfo{1, 1, K::R, K::HXA, K::TX, K::TY, K::SPT, K::PD, K::NT, K::SMEM,
                      &launch, &occupancy};
  }
};

// the row kernel of the conserved pattern (sp_chrow.cuh): grids of x extent
// NXR, periodic in x
template <class MF, int NXR, int YW, int SPT, int PD, bool QP, int MINB>
struct EntryChRow {
  using M = model_of<MF>;
  using K = ChRow<M, NXR, YW, SPT, PD, QP, MINB>;
  static constexpr auto kernel() {
    if constexpr (MINB > 1)
      return k_chrow_occ<M, K>;
    else
      return k_chrow<M, K>;
  }
  static cudaError_t launch(const void* prm, dim3 grid, cudaStream_t s) {
    auto kern = kernel();
    static cudaError_t attr = cudaFuncSetAttribute(
        kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(K::SMEM));
    if (attr != cudaSuccess) return attr;
    const M m = MF{}();
    return launch_step_kernel(kern, grid, K::NT, K::SMEM, s,
                              *static_cast<const StepParams<float>*>(prm), m);
  }
  static int occupancy() {
    auto kern = kernel();
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(K::SMEM));
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, K::NT, K::SMEM) != cudaSuccess)
      return 1;
    return n > 0 ? n : 1;
  }
  static KernelInfo info() {
    KernelInfo i{1, 1, K::R, K::HXA, K::TX, K::TY, K::SPT, K::PD, K::NT, K::SMEM,
                 &launch, &occupancy};
    i.box_hx = 0;
    i.nx_only = NXR;
    return i;
  }
};

// the row kernel of the fused 7-point models (sp_row.cuh): grids of x extent
// NXR, periodic in x
template <class MF, int NXR, int YW, int PD, int MINB>
struct EntryRow {
  using M = model_of<MF>;
  using K = RowCfg<M, NXR, YW, PD, MINB>;
  static constexpr auto kernel() {
    if constexpr (MINB > 1)
      return k_row_occ<M, K>;
    else
      return k_row<M, K>;
  }
  static cudaError_t launch(const void* prm, dim3 grid, cudaStream_t s) {
    auto kern = kernel();
    static cudaError_t attr = cudaFuncSetAttribute(
        kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(K::SMEM));
    if (attr != cudaSuccess) return attr;
    const M m = MF{}();
    return launch_step_kernel(kern, grid, K::NT, K::SMEM, s,
                              *static_cast<const StepParams<float>*>(prm), m);
  }
  static int occupancy() {
    auto kern = kernel();
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(K::SMEM));
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, K::NT, K::SMEM) != cudaSuccess)
      return 1;
    return n > 0 ? n : 1;
  }
  static KernelInfo info() {
    KernelInfo i{K::NF, K::NS, K::R, K::HXA, K::TX, K::TY, K::SPT, K::PD, K::NT, K::SMEM,
                 &launch, &occupancy};
    i.box_hx = 0;
    i.nx_only = NXR;
    return i;
  }
};

template <class MF0, class MF1, class T, int LP, int GP, int BP, class TC, bool EXACT>
struct Entry2 {
  using M0 = model_of<MF0>;
  using M1 = model_of<MF1>;
  using K = Fd2<M0, M1, T, LP, GP, BP, TC, EXACT>;
  static cudaError_t launch(const void* prm, dim3 grid, cudaStream_t s) {
    auto kern = k_fd2d<M0, M1, T, LP, GP, BP, TC, EXACT>;
    static cudaError_t attr = cudaFuncSetAttribute(
        kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(K::SMEM));
    if (attr != cudaSuccess) return attr;
    const M0 m0 = MF0{}();
    const M1 m1 = MF1{}();
    return launch_step_kernel(kern, grid, K::NT, K::SMEM, s,
                              *static_cast<const Step2Params<T>*>(prm), m0, m1);
  }
  static int occupancy() {
    auto kern = k_fd2d<M0, M1, T, LP, GP, BP, TC, EXACT>;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(K::SMEM));
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, K::NT, K::SMEM) != cudaSuccess)
      return 1;
    return n > 0 ? n : 1;
  }
  static KernelInfo info() {
    return KernelInfo{K::NF, K::NS,     K::R,    K::HXA,  K::TX,      K::TY,
                      K::SPT, K::PD, K::NT, K::SMEM, &launch, &occupancy};
  }
};

// the temporally blocked 2D step (sp_tb2.cuh): up to TC::KT steps per launch
template <class MF0, class MF1, class T, int LP, int GP, int BP, class TC, bool EXACT>
struct Entry2T {
  using M0 = model_of<MF0>;
  using M1 = model_of<MF1>;
  using K = Fd2T<M0, M1, T, LP, GP, BP, TC, EXACT>;
  static cudaError_t launch(const void* prm, dim3 grid, cudaStream_t s) {
    auto kern = k_fd2t<M0, M1, T, LP, GP, BP, TC, EXACT>;
    static cudaError_t attr = cudaFuncSetAttribute(
        kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(K::SMEM));
    if (attr != cudaSuccess) return attr;
    const M0 m0 = MF0{}();
    const M1 m1 = MF1{}();
    return launch_step_kernel(kern, grid, K::NT, K::SMEM, s,
                              *static_cast<const Step2Params<T>*>(prm), m0, m1);
  }
  static int occupancy() {
    auto kern = k_fd2t<M0, M1, T, LP, GP, BP, TC, EXACT>;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(K::SMEM));
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, K::NT, K::SMEM) != cudaSuccess)
      return 1;
    return n > 0 ? n : 1;
  }
  static KernelInfo info() {
    KernelInfo i{K::NF, K::NS, K::R, K::HXA, K::TX, K::TY, 1, 0, K::NT, K::SMEM,
                 &launch, &occupancy};
    i.kt = K::KT;
    i.x_multiple = K::LC;
    return i;
  }
};

// model factories
#define SP_FACTORY(NAME, EXPR)                          \
  struct NAME {                                         \
    constexpr auto operator()() const { return EXPR; } \
  };
SP_FACTORY(MF_A_exact, models::a_exact())
SP_FACTORY(MF_A_fused, models::a_fused())
SP_FACTORY(MF_B_exact, models::b_exact())
SP_FACTORY(MF_B_fused, models::b_fused())
SP_FACTORY(MF_C_exact, models::c_exact())
SP_FACTORY(MF_C_fused, models::c_fused())
SP_FACTORY(MF_AMK_exact, models::amk_exact())
SP_FACTORY(MF_AMK_fused, models::amk_fused())
SP_FACTORY(MF_BMK_exact, models::bmk_exact())
SP_FACTORY(MF_BMK_fused, models::bmk_fused())
SP_FACTORY(MF_OP_LAP, models::op_lap())
SP_FACTORY(MF_OP_BILAP, models::op_bilap())
SP_FACTORY(MF_OP_GRADLAP, models::op_gradlap())
SP_FACTORY(MF_OP_LAPCUBE, models::op_lapcube())
#undef SP_FACTORY

// a model factory whose models carry the halo reaches of stencils of order of
// accuracy ACC (Stencil2d4h: ACC = 4)
template <class MF, int ACC>
struct MFAcc {
  constexpr auto operator()() const { return ex::ModelAcc<decltype(MF{}()), ACC>{MF{}()}; }
};
using MF4_A_exact = MFAcc<MF_A_exact, 4>;
using MF4_B_exact = MFAcc<MF_B_exact, 4>;
using MF4_C_exact = MFAcc<MF_C_exact, 4>;
using MF4_AMK_exact = MFAcc<MF_AMK_exact, 4>;
using MF4_BMK_exact = MFAcc<MF_BMK_exact, 4>;
using MF4_OP_LAP = MFAcc<MF_OP_LAP, 4>;
using MF4_OP_BILAP = MFAcc<MF_OP_BILAP, 4>;
using MF4_OP_GRADLAP = MFAcc<MF_OP_GRADLAP, 4>;
using MF4_OP_LAPCUBE = MFAcc<MF_OP_LAPCUBE, 4>;

}  // namespace sp

// model ids and forms, as in include/symphas_b200.h
#define SPK_A 0
#define SPK_B 1
#define SPK_C 2
#define SPK_AMK 3
#define SPK_BMK 4
#define SPK_ENS_AB 5 /* 2D ensemble: instances of AMK and BMK in one launch */
#define SPK_OP_LAP 10
#define SPK_OP_BILAP 11
#define SPK_OP_GRADLAP 12
#define SPK_OP_LAPCUBE 13
#define SPK_EXACT 1
#define SPK_FUSED 0

// default tiles: 3D (TX, TY, rows per thread, planes in flight), 2D (.., tiles in flight)
namespace sp {
template <class T> struct Tiles;
template <> struct Tiles<float> {
  using D3 = TileCfg<64, 16, 4, 3, 2>;
  using D2 = TileCfg<128, 16, 4, 3, 2>;
  // further shapes the autotuner tries for the headline (fused FP32) kernels
  using D3b = TileCfg<64, 32, 4, 2, 2>;
  using D3c = TileCfg<128, 16, 4, 3, 2>;
  using D3d = TileCfg<128, 16, 4, 2, 2>;
  using D3e = TileCfg<64, 16, 2, 3, 2>;
  using D3f = TileCfg<64, 16, 4, 2, 2>;
  using C3a = TileCfg<64, 16, 4, 2, 2>;  // conserved-pattern kernel shapes
  using C3b = TileCfg<64, 16, 2, 2, 2>;
  using C3c = TileCfg<64, 32, 4, 2, 2>;
  using C3d = TileCfg<128, 16, 4, 2, 2>;
  // four x-sites per thread (16-byte shared-memory words)
  using D3w1 = TileCfg<128, 8, 2, 2, 4>;
  using D3w2 = TileCfg<128, 16, 4, 2, 4>;
  using D3w3 = TileCfg<64, 16, 2, 2, 4>;
  using D3w4 = TileCfg<128, 16, 2, 2, 4>;
  using D3w5 = TileCfg<64, 32, 4, 2, 4>;
  using D2w1 = TileCfg<128, 16, 4, 3, 4>;
  using D2w2 = TileCfg<128, 32, 4, 2, 4>;
  using D2w3 = TileCfg<128, 16, 2, 3, 4>;
  using D2b = TileCfg<64, 32, 4, 3, 2>;
  using D2c = TileCfg<128, 32, 8, 2, 2>;
  // fewer tiles in flight, less shared memory: more CTAs per SM
  using D2d = TileCfg<128, 16, 4, 2, 2>;
  using D2e = TileCfg<128, 16, 4, 1, 2>;
  // temporally blocked 2D tiles (sp_tb2.cuh): up to 2 and 4 steps per launch
  using T2a = TbCfg<128, 32, 2, 256, 4>;
  using T2b = TbCfg<128, 32, 4, 256, 4>;
};
template <> struct Tiles<double> {
  using D3 = TileCfg<64, 16, 2, 3, 2>;
  using D2 = TileCfg<64, 16, 4, 3, 2>;
  using T2a = TbCfg<64, 32, 2, 256, 2>;
};
}  // namespace sp

#define SP_REG3(MODEL, FORM, MF, T, DT, LP, GP, BP)                        \
  ::sp::register_kernel(::sp::KernelKey{MODEL, FORM, 3, DT, LP, GP, BP},    \
                        ::sp::Entry3<::sp::MF, T, LP, GP, BP, ::sp::Tiles<T>::D3, FORM == SPK_EXACT>::info())
#define SP_REG2(MODEL, FORM, MF, T, DT, LP, GP, BP)                        \
  ::sp::register_kernel(::sp::KernelKey{MODEL, FORM, 2, DT, LP, GP, BP},    \
                        ::sp::Entry2<::sp::MF, ::sp::MF, T, LP, GP, BP, ::sp::Tiles<T>::D2, FORM == SPK_EXACT>::info())
#define SP_REG3T(MODEL, FORM, MF, T, DT, LP, GP, BP, TILE)                  \
  ::sp::register_kernel(::sp::KernelKey{MODEL, FORM, 3, DT, LP, GP, BP},    \
                        ::sp::Entry3<::sp::MF, T, LP, GP, BP, TILE, FORM == SPK_EXACT>::info())
#define SP_REGCHROW(MODEL, MF, NXR, YW, SPT, PD, QP, MINB)                      \
  ::sp::register_kernel(::sp::KernelKey{MODEL, SPK_FUSED, 3, 0, 7, 10, 25},      \
                        ::sp::EntryChRow<::sp::MF, NXR, YW, SPT, PD, QP, MINB>::info())
#define SP_REGROW(MODEL, MF, NXR, YW, PD, MINB)                                 \
  ::sp::register_kernel(::sp::KernelKey{MODEL, SPK_FUSED, 3, 0, 7, 10, 25},      \
                        ::sp::EntryRow<::sp::MF, NXR, YW, PD, MINB>::info())
#define SP_REGCH3(MODEL, MF, TILE)                                          \
  ::sp::register_kernel(::sp::KernelKey{MODEL, SPK_FUSED, 3, 0, 7, 10, 25},  \
                        ::sp::EntryCh3<::sp::MF, float, TILE>::info())
#define SP_REG2T(MODEL, FORM, MF0, MF1, T, DT, LP, GP, BP, TILE)            \
  ::sp::register_kernel(::sp::KernelKey{MODEL, FORM, 2, DT, LP, GP, BP},    \
                        ::sp::Entry2<::sp::MF0, ::sp::MF1, T, LP, GP, BP, TILE, FORM == SPK_EXACT>::info())
#define SP_REG2TB(MODEL, FORM, MF0, MF1, T, DT, LP, GP, BP, TILE)           \
  ::sp::register_kernel(::sp::KernelKey{MODEL, FORM, 2, DT, LP, GP, BP},    \
                        ::sp::Entry2T<::sp::MF0, ::sp::MF1, T, LP, GP, BP, TILE, FORM == SPK_EXACT>::info())
#define SP_REG2X(MODEL, FORM, MF0, MF1, T, DT, LP, GP, BP)                 \
  ::sp::register_kernel(::sp::KernelKey{MODEL, FORM, 2, DT, LP, GP, BP},    \
                        ::sp::Entry2<::sp::MF0, ::sp::MF1, T, LP, GP, BP, ::sp::Tiles<T>::D2, FORM == SPK_EXACT>::info())
