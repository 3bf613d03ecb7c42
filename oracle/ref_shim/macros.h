// Minimal stand-in for cuda-utils' macros.h (written for this project); ASSERT comes from the
// cuda_utils.h stand-in. Test infrastructure only.
#pragma once
