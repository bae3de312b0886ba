/*
 * sp_inst_wide.cu -- FP32 fused-form kernels with four x-sites per thread
 * (16-byte shared-memory words, two packed FP32x2 instructions per
 * operation).  They evaluate every site exactly as the two-site kernels do
 * and share their field layout, so they are further tile shapes for
 * sp_autotune (registered after the fused set, in their own translation unit
 * so that the build compiles them in parallel), together with the row kernels
 * of the conserved pattern (sp_chrow.cuh) and of any fused 7-point model
 * (sp_row.cuh).
 */
#include "sp_launch.cuh"

#define SP_WIDE3(MODEL, MF)                                                         \
  SP_REG3T(MODEL, SPK_FUSED, MF, float, 0, 7, 10, 25, ::sp::Tiles<float>::D3w1);   \
  SP_REG3T(MODEL, SPK_FUSED, MF, float, 0, 7, 10, 25, ::sp::Tiles<float>::D3w2);   \
  SP_REG3T(MODEL, SPK_FUSED, MF, float, 0, 7, 10, 25, ::sp::Tiles<float>::D3w3);   \
  SP_REG3T(MODEL, SPK_FUSED, MF, float, 0, 7, 10, 25, ::sp::Tiles<float>::D3w4);   \
  SP_REG3T(MODEL, SPK_FUSED, MF, float, 0, 7, 10, 25, ::sp::Tiles<float>::D3w5);
#define SP_WIDE2(MODEL, MF0, MF1)                                                   \
  SP_REG2T(MODEL, SPK_FUSED, MF0, MF1, float, 0, 5, 6, 13, ::sp::Tiles<float>::D2w1); \
  SP_REG2T(MODEL, SPK_FUSED, MF0, MF1, float, 0, 5, 6, 13, ::sp::Tiles<float>::D2w2); \
  SP_REG2T(MODEL, SPK_FUSED, MF0, MF1, float, 0, 5, 6, 13, ::sp::Tiles<float>::D2w3); \
  SP_REG2T(MODEL, SPK_FUSED, MF0, MF1, float, 0, 5, 6, 13, ::sp::Tiles<float>::D2d);  \
  SP_REG2T(MODEL, SPK_FUSED, MF0, MF1, float, 0, 5, 6, 13, ::sp::Tiles<float>::D2e);

namespace sp {
void register_wide_kernels() {
  SP_WIDE3(SPK_A, MF_A_fused)
  SP_WIDE3(SPK_B, MF_B_fused)
  SP_WIDE3(SPK_C, MF_C_fused)
  // row kernels of the conserved pattern (x extent 256 or 128, periodic in x)
  SP_REGCHROW(SPK_B, MF_B_fused, 256, 10, 1, 2, true, 2);
  SP_REGCHROW(SPK_B, MF_B_fused, 256, 10, 1, 2, false, 2);
  SP_REGCHROW(SPK_B, MF_B_fused, 256, 18, 1, 2, true, 1);
  SP_REGCHROW(SPK_B, MF_B_fused, 256, 6, 1, 2, false, 1);
  SP_REGCHROW(SPK_B, MF_B_fused, 256, 6, 1, 2, true, 1);
  SP_REGCHROW(SPK_B, MF_B_fused, 256, 6, 1, 3, false, 1);
  SP_REGCHROW(SPK_B, MF_B_fused, 256, 3, 2, 2, false, 1);
  SP_REGCHROW(SPK_B, MF_B_fused, 128, 9, 2, 2, true, 1);
  SP_REGCHROW(SPK_B, MF_B_fused, 128, 18, 1, 2, true, 1);
  SP_REGCHROW(SPK_BMK, MF_BMK_fused, 256, 10, 1, 2, true, 2);
  // row kernels of any fused 7-point model (sp_row.cuh)
  SP_REGROW(SPK_C, MF_C_fused, 256, 6, 1, 1);
  SP_REGROW(SPK_C, MF_C_fused, 256, 6, 2, 1);
  SP_REGROW(SPK_C, MF_C_fused, 256, 10, 1, 1);
  SP_REGROW(SPK_C, MF_C_fused, 128, 10, 2, 1);
  SP_REGROW(SPK_A, MF_A_fused, 256, 8, 2, 1);
  SP_REGROW(SPK_A, MF_A_fused, 128, 16, 2, 1);
  SP_REGROW(SPK_B, MF_B_fused, 256, 10, 2, 2);
  SP_REGCHROW(SPK_BMK, MF_BMK_fused, 128, 9, 2, 2, true, 1);
  SP_WIDE2(SPK_A, MF_A_fused, MF_A_fused)
  SP_WIDE2(SPK_B, MF_B_fused, MF_B_fused)
  SP_WIDE2(SPK_ENS_AB, MF_AMK_fused, MF_BMK_fused)
}
}  // namespace sp
