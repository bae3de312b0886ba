/*
 * sp_inst_exact.cu -- kernels of the EXACT form (the reference's printed term
 * order).  This unit is compiled with --fmad=false so every product and sum
 * rounds on its own, as in the CPU solver; in FP64 the fields then agree with
 * SymPhas's SolverFT bit for bit.
 */
#include "sp_launch.cuh"

#define SP_EXACT_SET(T, DT, L2, G2, B2, L3, G3, B3)                     \
  SP_REG2(SPK_A, SPK_EXACT, MF_A_exact, T, DT, L2, G2, B2);                        \
  SP_REG2(SPK_B, SPK_EXACT, MF_B_exact, T, DT, L2, G2, B2);                        \
  SP_REG2(SPK_C, SPK_EXACT, MF_C_exact, T, DT, L2, G2, B2);                        \
  SP_REG2(SPK_AMK, SPK_EXACT, MF_AMK_exact, T, DT, L2, G2, B2);                    \
  SP_REG2(SPK_BMK, SPK_EXACT, MF_BMK_exact, T, DT, L2, G2, B2);                    \
  SP_REG2X(SPK_ENS_AB, SPK_EXACT, MF_AMK_exact, MF_BMK_exact, T, DT, L2, G2, B2);  \
  SP_REG3(SPK_A, SPK_EXACT, MF_A_exact, T, DT, L3, G3, B3);                        \
  SP_REG3(SPK_B, SPK_EXACT, MF_B_exact, T, DT, L3, G3, B3);                        \
  SP_REG3(SPK_C, SPK_EXACT, MF_C_exact, T, DT, L3, G3, B3);                        \
  SP_REG3(SPK_AMK, SPK_EXACT, MF_AMK_exact, T, DT, L3, G3, B3);                    \
  SP_REG3(SPK_BMK, SPK_EXACT, MF_BMK_exact, T, DT, L3, G3, B3);                    \
  SP_REG2(SPK_OP_LAPCUBE, SPK_EXACT, MF_OP_LAPCUBE, T, DT, L2, G2, B2);            \
  SP_REG3(SPK_OP_LAPCUBE, SPK_EXACT, MF_OP_LAPCUBE, T, DT, L3, G3, B3);

// single-operator kernels for every point set of Stencil2d2h / Stencil3d2h
#define SP_OPS2(T, DT)                                         \
  SP_REG2(SPK_OP_LAP, SPK_EXACT, MF_OP_LAP, T, DT, 5, 6, 13);  \
  SP_REG2(SPK_OP_LAP, SPK_EXACT, MF_OP_LAP, T, DT, 9, 6, 13);  \
  SP_REG2(SPK_OP_BILAP, SPK_EXACT, MF_OP_BILAP, T, DT, 5, 6, 13); \
  SP_REG2(SPK_OP_BILAP, SPK_EXACT, MF_OP_BILAP, T, DT, 5, 6, 17); \
  SP_REG2(SPK_OP_BILAP, SPK_EXACT, MF_OP_BILAP, T, DT, 5, 6, 21); \
  SP_REG2(SPK_OP_GRADLAP, SPK_EXACT, MF_OP_GRADLAP, T, DT, 5, 6, 13);  \
  SP_REG2(SPK_OP_GRADLAP, SPK_EXACT, MF_OP_GRADLAP, T, DT, 5, 8, 13);  \
  SP_REG2(SPK_OP_GRADLAP, SPK_EXACT, MF_OP_GRADLAP, T, DT, 5, 12, 13); \
  SP_REG2(SPK_OP_GRADLAP, SPK_EXACT, MF_OP_GRADLAP, T, DT, 5, 16, 13);
#define SP_OPS3(T, DT)                                          \
  SP_REG3(SPK_OP_LAP, SPK_EXACT, MF_OP_LAP, T, DT, 7, 10, 25);  \
  SP_REG3(SPK_OP_LAP, SPK_EXACT, MF_OP_LAP, T, DT, 15, 10, 25); \
  SP_REG3(SPK_OP_LAP, SPK_EXACT, MF_OP_LAP, T, DT, 19, 10, 25); \
  SP_REG3(SPK_OP_LAP, SPK_EXACT, MF_OP_LAP, T, DT, 21, 10, 25); \
  SP_REG3(SPK_OP_LAP, SPK_EXACT, MF_OP_LAP, T, DT, 27, 10, 25); \
  SP_REG3(SPK_OP_BILAP, SPK_EXACT, MF_OP_BILAP, T, DT, 7, 10, 21); \
  SP_REG3(SPK_OP_BILAP, SPK_EXACT, MF_OP_BILAP, T, DT, 7, 10, 25); \
  SP_REG3(SPK_OP_BILAP, SPK_EXACT, MF_OP_BILAP, T, DT, 7, 10, 41); \
  SP_REG3(SPK_OP_BILAP, SPK_EXACT, MF_OP_BILAP, T, DT, 7, 10, 52); \
  SP_REG3(SPK_OP_BILAP, SPK_EXACT, MF_OP_BILAP, T, DT, 7, 10, 57); \
  SP_REG3(SPK_OP_GRADLAP, SPK_EXACT, MF_OP_GRADLAP, T, DT, 7, 10, 25); \
  SP_REG3(SPK_OP_GRADLAP, SPK_EXACT, MF_OP_GRADLAP, T, DT, 7, 12, 25); \
  SP_REG3(SPK_OP_GRADLAP, SPK_EXACT, MF_OP_GRADLAP, T, DT, 7, 28, 25); \
  SP_REG3(SPK_OP_GRADLAP, SPK_EXACT, MF_OP_GRADLAP, T, DT, 7, 36, 25); \
  SP_REG3(SPK_OP_GRADLAP, SPK_EXACT, MF_OP_GRADLAP, T, DT, 7, 40, 25);

// Stencil2d4h (2D, 4th order): the models with SymPhas's default point sets
// Stencil2d4h<> = <9,14,21> (sol/inc/stencilincludes.h:774-779), and each
// operator with every point set of sol/inc/stencilh4.h
#define SP_EXACT_SET4(T, DT)                                                           \
  SP_REG2(SPK_A, SPK_EXACT, MF4_A_exact, T, DT, 1009, 1014, 1021);                      \
  SP_REG2(SPK_B, SPK_EXACT, MF4_B_exact, T, DT, 1009, 1014, 1021);                      \
  SP_REG2(SPK_C, SPK_EXACT, MF4_C_exact, T, DT, 1009, 1014, 1021);                      \
  SP_REG2(SPK_AMK, SPK_EXACT, MF4_AMK_exact, T, DT, 1009, 1014, 1021);                  \
  SP_REG2(SPK_BMK, SPK_EXACT, MF4_BMK_exact, T, DT, 1009, 1014, 1021);                  \
  SP_REG2(SPK_OP_LAPCUBE, SPK_EXACT, MF4_OP_LAPCUBE, T, DT, 1009, 1014, 1021);
#define SP_OPS2_4(T, DT)                                                               \
  SP_REG2(SPK_OP_LAP, SPK_EXACT, MF4_OP_LAP, T, DT, 1009, 1014, 1021);                  \
  SP_REG2(SPK_OP_LAP, SPK_EXACT, MF4_OP_LAP, T, DT, 1017, 1014, 1021);                  \
  SP_REG2(SPK_OP_LAP, SPK_EXACT, MF4_OP_LAP, T, DT, 1021, 1014, 1021);                  \
  SP_REG2(SPK_OP_BILAP, SPK_EXACT, MF4_OP_BILAP, T, DT, 1009, 1014, 1021);              \
  SP_REG2(SPK_OP_BILAP, SPK_EXACT, MF4_OP_BILAP, T, DT, 1009, 1014, 1025);              \
  SP_REG2(SPK_OP_BILAP, SPK_EXACT, MF4_OP_BILAP, T, DT, 1009, 1014, 1033);              \
  SP_REG2(SPK_OP_BILAP, SPK_EXACT, MF4_OP_BILAP, T, DT, 1009, 1014, 1037);              \
  SP_REG2(SPK_OP_GRADLAP, SPK_EXACT, MF4_OP_GRADLAP, T, DT, 1009, 1014, 1021);          \
  SP_REG2(SPK_OP_GRADLAP, SPK_EXACT, MF4_OP_GRADLAP, T, DT, 1009, 1018, 1021);          \
  SP_REG2(SPK_OP_GRADLAP, SPK_EXACT, MF4_OP_GRADLAP, T, DT, 1009, 1026, 1021);          \
  SP_REG2(SPK_OP_GRADLAP, SPK_EXACT, MF4_OP_GRADLAP, T, DT, 1009, 1030, 1021);

namespace sp {
void register_exact_kernels() {
  SP_EXACT_SET4(double, 1)
  SP_EXACT_SET4(float, 0)
  SP_OPS2_4(double, 1)
  // the benchmarked point sets <5,6,13> / <7,10,25> and SymPhas's defaults (Stencil2d2h<> = <9,6,13>,
  // Stencil3d2h<> = <15,10,25>, sol/inc/stencilincludes.h:758-792, 884-921)
  SP_EXACT_SET(double, 1, 5, 6, 13, 7, 10, 25)
  SP_EXACT_SET(double, 1, 9, 6, 13, 15, 10, 25)
  SP_EXACT_SET(float, 0, 5, 6, 13, 7, 10, 25)
  SP_EXACT_SET(float, 0, 9, 6, 13, 15, 10, 25)
  SP_OPS2(double, 1)
  SP_OPS3(double, 1)
  // temporally blocked FP64 shapes (sp_tb2.cuh), two steps per launch: the
  // same bits as two one-step launches
  SP_REG2TB(SPK_A, SPK_EXACT, MF_A_exact, MF_A_exact, double, 1, 5, 6, 13, ::sp::Tiles<double>::T2a);
  SP_REG2TB(SPK_B, SPK_EXACT, MF_B_exact, MF_B_exact, double, 1, 5, 6, 13, ::sp::Tiles<double>::T2a);
  SP_REG2TB(SPK_C, SPK_EXACT, MF_C_exact, MF_C_exact, double, 1, 5, 6, 13, ::sp::Tiles<double>::T2a);
  SP_REG2TB(SPK_ENS_AB, SPK_EXACT, MF_AMK_exact, MF_BMK_exact, double, 1, 5, 6, 13,
            ::sp::Tiles<double>::T2a);
}
}  // namespace sp
