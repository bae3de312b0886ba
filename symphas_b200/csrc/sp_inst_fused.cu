/*
 * sp_inst_fused.cu -- kernels of the FUSED form (bilap = lap o lap, merged
 * derivatives, staged operands); FMA contraction allowed.  For point sets
 * where bilap is not lap o lap, the FUSED key runs the exact term order
 * compiled with FMA.
 */
#include "sp_launch.cuh"

#define SP_FUSED_SET(T, DT)                                                \
  SP_REG2(SPK_A, SPK_FUSED, MF_A_fused, T, DT, 5, 6, 13);                            \
  SP_REG2(SPK_B, SPK_FUSED, MF_B_fused, T, DT, 5, 6, 13);                            \
  SP_REG2(SPK_C, SPK_FUSED, MF_C_fused, T, DT, 5, 6, 13);                            \
  SP_REG2(SPK_AMK, SPK_FUSED, MF_AMK_fused, T, DT, 5, 6, 13);                        \
  SP_REG2(SPK_BMK, SPK_FUSED, MF_BMK_fused, T, DT, 5, 6, 13);                        \
  SP_REG2X(SPK_ENS_AB, SPK_FUSED, MF_AMK_fused, MF_BMK_fused, T, DT, 5, 6, 13);      \
  SP_REG3(SPK_A, SPK_FUSED, MF_A_fused, T, DT, 7, 10, 25);                           \
  SP_REG3(SPK_B, SPK_FUSED, MF_B_fused, T, DT, 7, 10, 25);                           \
  SP_REG3(SPK_C, SPK_FUSED, MF_C_fused, T, DT, 7, 10, 25);                           \
  SP_REG3(SPK_AMK, SPK_FUSED, MF_AMK_fused, T, DT, 7, 10, 25);                       \
  SP_REG3(SPK_BMK, SPK_FUSED, MF_BMK_fused, T, DT, 7, 10, 25);                       \
  SP_REG2(SPK_A, SPK_FUSED, MF_A_fused, T, DT, 9, 6, 13);                            \
  SP_REG2(SPK_B, SPK_FUSED, MF_B_exact, T, DT, 9, 6, 13);                            \
  SP_REG2(SPK_C, SPK_FUSED, MF_C_exact, T, DT, 9, 6, 13);                            \
  SP_REG3(SPK_A, SPK_FUSED, MF_A_fused, T, DT, 15, 10, 25);                          \
  SP_REG3(SPK_B, SPK_FUSED, MF_B_exact, T, DT, 15, 10, 25);                          \
  SP_REG3(SPK_C, SPK_FUSED, MF_C_exact, T, DT, 15, 10, 25);

namespace sp {
void register_fused_kernels() {
  SP_FUSED_SET(float, 0)
  SP_FUSED_SET(double, 1)
}
}  // namespace sp
