// Runtime compilation (NVRTC) of the step kernels with a user yield
// function generated as straight-line code (expr.cpp: emitYieldPolicy).
#pragma once

#include <string>
#include <vector>

#include "engine.hpp"

namespace dl {

// Kernels of step.cuh instantiated with the generated policy for precision
// float (fp32) or double on the current device; compiled once per process
// (and cached on disk under $DL_JIT_CACHE, default ~/.cache/dynlattice_b200).
// Returns nullptr with a message in *log when NVRTC is unavailable or fails.
const KernelSet *jit_kernels(const std::string &policy_source, bool fp32, std::string *log);

// Compile only (no device needed): cubin for sm_100a and the lowered kernel names.
bool jit_compile(const std::string &policy_source, bool fp32, std::vector<char> *cubin,
                 std::vector<std::string> *lowered, std::string *log);

// Adjoint kernels (adjoint_kernels.cuh) with the generated YieldAdj policy
// (expr.cpp: emitYieldAdjPolicy); same caching as jit_kernels.
const AdjKernels *jit_adjoint_kernels(const std::string &adj_policy_source, bool fp32, std::string *log);
bool jit_compile_adjoint(const std::string &adj_policy_source, bool fp32, std::vector<char> *cubin,
                         std::vector<std::string> *lowered, std::string *log);

}  // namespace dl
