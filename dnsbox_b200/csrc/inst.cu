// Explicit instantiation of the pass kernels for one (precision, size) pair.
// Built once per pair with -DINST_T=<double|float> -DINST_N=<n>.
#define DNSBOX_LAUNCH_IMPL
#include "launch.cuh"

#ifndef INST_T
#error "INST_T must be defined"
#endif
#ifndef INST_N
#error "INST_N must be defined"
#endif

namespace dnsbox {
template struct Launcher<INST_T, INST_N>;
}
