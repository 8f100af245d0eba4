// Test infrastructure only: the reference's LUonDevice provided by the B200
// engine's header-only shim, so that the reference's own lu_cmd.cpp and
// symbolic.cc link against libglu_b200.so instead of numeric.cu (drop-in check).
#include "symbolic.h"
#define GLU_PROVIDE_LUONDEVICE
#include "glu_luondevice.hpp"
#include "numeric.h"
