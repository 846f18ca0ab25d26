/* uk_pb.cu -- the user-kernel launchers of one precision (-DUK_PB=<bits>),
 * compiled once per precision (see user_kernels.cuh). */
#include "user_kernels.cuh"

#ifndef UK_PB
#error "build with -DUK_PB=<precision in bits>"
#endif

namespace uk {
#if UK_PB > 2048
UK_REAL_LAUNCHERS(, UK_PB)
#else
UK_LAUNCHERS(, UK_PB)
#endif
#if UK_PB < 2048 /* the elementary functions stop below 2048 bits (constant tables) */
UK_FN_LAUNCHERS(, UK_PB)
#endif
}  // namespace uk
