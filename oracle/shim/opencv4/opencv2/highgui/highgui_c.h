/* Test-only: forwards to the OpenCV C-API declarations in core_c.h. */
#include "../core/core_c.h"
