// Stand-in for cuRAND's device API (test infrastructure): curand_uniform
// returns the values queued by the golden-vector driver, in order, so the
// reference's own sampling code can be driven with known draws.
#ifndef R2_REFSHIM_CURAND_KERNEL_H
#define R2_REFSHIM_CURAND_KERNEL_H
#include <cstdint>
struct curandStateXORWOW { int unused; };
typedef curandStateXORWOW curandState_t;
namespace r2ref {
float next_curand();
}
inline float curand_uniform(curandState_t*) { return r2ref::next_curand(); }
inline void curand_init(unsigned long long, unsigned long long, unsigned long long, curandState_t*) {}
#endif
