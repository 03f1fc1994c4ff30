/* svpf.cuh -- the reference's header name (include/svpf.cuh), kept so that its
 * callers (tests, tools, svpf_multiscale.cuh-style compositions) compile
 * unchanged against this engine.  Everything is declared in svpf.h. */
#ifndef SVPF_B200_CUH_SHIM
#define SVPF_B200_CUH_SHIM
#include "svpf.h"
#endif
