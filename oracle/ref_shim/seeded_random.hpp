/* Pre-included into the reference checker build -- TEST INFRASTRUCTURE ONLY.
 * The reference's generateArrayRandom1D seeds std::default_random_engine from
 * std::random_device (include/utils/TestTools/generateTools.hpp:79-102), which
 * makes its Lanczos start vector irreproducible.  This header takes that
 * header's include guard and provides the one function of it the compiled
 * sources use, with the same engine and distribution but a seed taken from
 * prism_ref_next_seed() (base seed + call index, set by the checker). */
#ifndef CUDATOOLS_GENERATE_TOOLS_H
#define CUDATOOLS_GENERATE_TOOLS_H
#include "config/headers.h"
#include "config/config.h"
#include "config/debug.h"
extern "C" unsigned prism_ref_next_seed(void);
namespace HOST {
template <typename T>
void generateArrayRandom1D(T* values, UINT32 size) {
    std::default_random_engine generator(prism_ref_next_seed());
    std::uniform_real_distribution<FLOAT32> distribution(-1.0, 1.0);
    for (UINT32 i = 0; i < size; i++) values[i] = distribution(generator);
}
}  // namespace HOST
#endif
