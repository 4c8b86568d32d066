/* Force-included (gcc -include) into every translation unit of the reference
 * build under oracle/_ref.  It is test infrastructure, never product code.
 *
 * The reference reads heap memory it never wrote: the Laplacian buffer `wave`
 * of fdm2d/fdm (pywave/src/wave_fdm.c:150,496) keeps its two outer rows and
 * columns unwritten (stencil loop wave_fdm.c:574-575) yet the leapfrog update
 * reads them (wave_fdm.c:590-601); `term` in forward_modeling_a
 * (wave_fwimodeling.c:55) and the first-shot forward of gradient_av
 * (wave_fwigradient.c:114) have the same defect.  With plain malloc the
 * reference output depends on whatever the allocator returns.  Zero-filled
 * allocation turns those reads into the value the algorithm evidently means
 * (an exact zero border), which is the semantics the CUDA kernels implement.
 */
#ifndef PW_ORACLE_ZERO_MALLOC_H
#define PW_ORACLE_ZERO_MALLOC_H
#include <stdlib.h>
#define malloc(n) calloc(1, (n))
#endif
