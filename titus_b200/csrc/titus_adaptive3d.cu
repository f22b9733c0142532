// The rank-adaptive BUG integrator on 3D problems (titus_create_3d): the
// kernels and host code of titus_adaptive.cu compiled with six streaming pairs
// -- (L2x, Ax), (L2y, Az), (L1x, |Ax|), (L1y, |Az|), (L2z, Ay), (L1z, |Ay|) --
// the 3D boundary test, the z term of the uncollided sweep, and their own
// namespace (titus::wide3) and host entry names (*_3d). Everything else (the
// augmentation, range finders, truncation, rejection tests, scattering steps)
// is the same code as the 2D build.
#define TITUS_WIDE_NOPS 6
#define TITUS_WIDE_NS wide3
#define TITUS_WIDE_HOST(name) name##_3d
#include "titus_adaptive.cu"
