/* The reference includes the pre-v3 NVTX header name. */
#pragma once
#include <nvtx3/nvToolsExt.h>
