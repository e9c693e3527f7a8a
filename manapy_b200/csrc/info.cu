// Build information of the library.
#include "manapy_b200.h"

#define MB_STR2(x) #x
#define MB_STR(x) MB_STR2(x)

extern "C" const char *mb_build_info(void) {
  return "manapy_b200 sm_100a fp64 nvcc " MB_STR(__CUDACC_VER_MAJOR__) "." MB_STR(__CUDACC_VER_MINOR__);
}
