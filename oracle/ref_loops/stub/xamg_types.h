// Stand-in for the reference's src/xamg_types.h, found before it on the
// include path: the reference's misc/rand.h needs only the floating-point
// typedefs and the alignment macros from it, not the logging and
// performance-counter headers it pulls in.
#pragma once
#include <cstdint>
typedef float float32_t;
typedef double float64_t;
#define XAMG_ALIGN_SIZE 64
#define XAMG_STACK_ALIGNMENT_PREFIX alignas(XAMG_ALIGN_SIZE)
