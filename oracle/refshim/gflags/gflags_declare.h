/* see gflags.h in this folder */
#pragma once
#include "gflags.h"
