// Host stand-in for <cuda_fp16.h>; the prelude already defines half.
#pragma once
#include "ab_ref_prelude.h"
