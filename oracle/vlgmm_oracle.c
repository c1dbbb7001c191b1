/* Oracle library: the C restatement of the GMM-EM / Fisher-vector path in
 * float and double.  TEST INFRASTRUCTURE ONLY (see vlgmm_oracle_impl.h). */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stddef.h>

#define ORC_PI 3.141592653589793
/* Fisher flags, same bit values as vl/fisher.h:23-26. */
#define ORC_FLAG_SQUARE_ROOT (1 << 0)
#define ORC_FLAG_NORMALIZED (1 << 1)
#define ORC_FLAG_FAST (1 << 2)

#define REAL float
#define SFX _f
#include "vlgmm_oracle_impl.h"
#undef REAL
#undef SFX

#define REAL double
#define SFX _d
#include "vlgmm_oracle_impl.h"
#undef REAL
#undef SFX
