// Compiled and run by tests/test_abi_macros.py.  Includes ppm_b200.h the way an Enzo
// source file does, after macros_and_parameters.h has put Enzo's LARGE_INTS and
// CONFIG_BFLOAT_8 macros in force (macros_and_parameters.h:151, :217, :257), then asks
// the library whether the structs this translation unit sees have the library's layout
// and calls entry points through the prototypes it declared.  System headers come
// first, as in Enzo's sources (Grid_SolvePPM_DE.C:20-22).
#include <stddef.h>
typedef long long long_int;
#define int long_int
#define float double
#include "ppm_b200.h"

// the header gives the macros back to the code that follows it
static_assert(sizeof(int) == sizeof(long long), "Enzo's int macro is in force after the header");
static_assert(sizeof(float) == sizeof(double), "Enzo's float macro is in force after the header");

static const long long kLayout[] = {PPM_B200_ABI_LAYOUT(PPM_B200_ABI_ITEM)};
static const long long kCount = sizeof(kLayout) / sizeof(kLayout[0]);

// calls made while Enzo's macros are in force, as Enzo's own code would make them
static long_int check_layout() { return ppm_b200_abi_check(kLayout, kCount); }
static long_int version() { return ppm_b200_version(); }
static const char* unsupported_message() { return ppm_b200_error_string(PPM_B200_ERR_UNSUPPORTED); }
static long_int params_size() { return sizeof(ppm_b200_params); }

#undef int
#undef float
#include <cstdio>
#include <cstring>

int main() {
  const long long rc = check_layout();
  const long long v = version();
  const char* msg = unsupported_message();
  std::printf("abi_check=%lld version=%lld params_bytes=%lld entries=%lld\n", rc, v,
              (long long)params_size(), kCount);
  if (rc != PPM_B200_OK) return 1;
  if (v != PPM_B200_VERSION) return 2;
  if (std::strncmp(msg, "configuration", 13) != 0) return 3;
  return 0;
}
