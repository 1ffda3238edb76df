// kw_inst.cu -- the kernel launchers of one axis length.
//
// Compiled once per compile-time axis length with -DKW_INST_N=<length>, and
// once with -DKW_INST_N=0 for the runtime-radix kernels, so the transform and
// stage kernels of the different lengths compile in parallel.
#include "kw_launch.cuh"

#ifndef KW_INST_N
#error "compile kw_inst.cu with -DKW_INST_N=<axis length, or 0 for the runtime-radix kernels>"
#endif

namespace kw {
template struct YLaunch<KW_INST_N>;
template struct XLaunch<KW_INST_N>;
template struct ZR2CLaunch<KW_INST_N>;
template struct ZC2RLaunch<KW_INST_N>;
template struct ULaunch<KW_INST_N>;
template struct RLaunch<KW_INST_N>;
template struct PLaunch<KW_INST_N>;
}  // namespace kw
