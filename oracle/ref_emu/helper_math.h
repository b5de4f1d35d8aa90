/*
 * helper_math.h -- TEST INFRASTRUCTURE ONLY.
 *
 * The reference includes <helper_math.h>, a CUDA-samples header that its
 * build downloads at configure time (src/CMakeLists.txt:11-13) and that is
 * not part of the reference sources.  Of that header, the DEM kernels use
 * only the integer vector sum in src/contactsearch.cuh:361 and :584
 * (gridPos + make_int3(...)), which is defined here.
 */
#ifndef SPHERE_REF_HELPER_MATH_STANDIN_H_
#define SPHERE_REF_HELPER_MATH_STANDIN_H_

#include <vector_types.h>

inline int3 operator+(int3 a, int3 b)
{
    int3 r;
    r.x = a.x + b.x;
    r.y = a.y + b.y;
    r.z = a.z + b.z;
    return r;
}

#endif
