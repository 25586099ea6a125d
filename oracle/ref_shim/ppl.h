/* POSIX stand-in for the PPL parallel_for used by the reference engine, mapped onto an
 * OpenMP loop with one iteration per worker (oracle test infrastructure only). */
#pragma once
#include <omp.h>
namespace Concurrency {
template <typename F> void parallel_for(int first, int last, F f) {
    #pragma omp parallel for schedule(dynamic, 1)
    for (int i = first; i < last; i++) f(i);
}
}
