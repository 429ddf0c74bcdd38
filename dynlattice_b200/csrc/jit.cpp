// NVRTC compilation of the step kernels (see jit.hpp).
#include "jit.hpp"

#include <cuda_runtime.h>
#include <nvrtc.h>

#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <map>
#include <memory>
#include <mutex>
#include <sstream>
#include <sys/stat.h>
#include <vector>

#include "jit_sources.inc"  // kJitHeaderNames / kJitHeaders (generated from the .cuh files)

namespace dl {

namespace {

constexpr int kNames = 10;

struct Entry {
  cudaLibrary_t lib = nullptr;
  KernelSet ks;
};

std::mutex g_mu;
std::map<std::string, std::unique_ptr<Entry>> g_cache;

uint64_t fnv1a(const std::string &s) {
  uint64_t h = 1469598103934665603ULL;
  for (unsigned char c : s) {
    h ^= c;
    h *= 1099511628211ULL;
  }
  return h;
}

std::string cache_dir() {
  const char *d = std::getenv("DL_JIT_CACHE");
  if (d && *d) return d;
  const char *home = std::getenv("HOME");
  return std::string(home ? home : "/tmp") + "/.cache/dynlattice_b200";
}

void mkdirs(const std::string &p) {
  std::string cur;
  std::stringstream ss(p);
  std::string part;
  if (!p.empty() && p[0] == '/') cur = "/";
  while (std::getline(ss, part, '/')) {
    if (part.empty()) continue;
    cur += part + "/";
    mkdir(cur.c_str(), 0755);
  }
}

bool read_file(const std::string &path, std::vector<char> &out) {
  std::ifstream f(path, std::ios::binary);
  if (!f) return false;
  out.assign(std::istreambuf_iterator<char>(f), std::istreambuf_iterator<char>());
  return !out.empty();
}

}  // namespace

namespace {

// compile `src` (which includes the embedded headers) for sm_100a and lower
// the kernel name expressions; results cached on disk by content hash
bool compile_generic(const std::string &src, const std::vector<std::string> &names, bool fp32,
                     const std::string &tag, std::vector<char> *cubin, std::vector<std::string> *lowered,
                     std::string *log) {
  const char *T = fp32 ? "float" : "double";
  // the FP32 variant uses approximate (not correctly rounded) division and
  // square root; transcendentals stay accurate (small rotation angles need a
  // relative error bound).  Its error budget against the FP64 path is 1e-5.
  const char *opts32[] = {"-arch=sm_100a", "-std=c++17", "-DNDEBUG", "-prec-div=false", "-prec-sqrt=false",
                          "-ftz=true"};
  const char *opts64[] = {"-arch=sm_100a", "-std=c++17", "-DNDEBUG"};
  const char *const *opts = fp32 ? opts32 : opts64;
  const int nopts = fp32 ? 6 : 3;
  const int nk = static_cast<int>(names.size());
  int nv_major = 0, nv_minor = 0;
  nvrtcVersion(&nv_major, &nv_minor);
  std::string full = src + (fp32 ? "|approx-div-sqrt" : "");
  for (auto &n : names) full += "|" + n;
  for (size_t i = 0; i < sizeof(kJitHeaders) / sizeof(kJitHeaders[0]); ++i) full += kJitHeaders[i];
  char hbuf[64];
  std::snprintf(hbuf, sizeof hbuf, "%016llx_%d_%d_%s", static_cast<unsigned long long>(fnv1a(full)), nv_major,
                nv_minor, T);
  const std::string dir = cache_dir();
  const std::string cubin_path = dir + "/" + tag + "_" + hbuf + ".cubin";
  const std::string names_path = dir + "/" + tag + "_" + hbuf + ".names";
  lowered->assign(nk, "");
  {
    std::vector<char> nb;
    if (read_file(cubin_path, *cubin) && read_file(names_path, nb)) {
      std::stringstream ns(std::string(nb.begin(), nb.end()));
      for (int i = 0; i < nk; ++i) std::getline(ns, (*lowered)[i]);
      if (!(*lowered)[nk - 1].empty()) return true;
    }
  }
  nvrtcProgram prog;
  const int nh = static_cast<int>(sizeof(kJitHeaders) / sizeof(kJitHeaders[0]));
  if (nvrtcCreateProgram(&prog, src.c_str(), "dl_jit.cu", nh, kJitHeaders, kJitHeaderNames) != NVRTC_SUCCESS) {
    if (log) *log = "nvrtcCreateProgram failed";
    return false;
  }
  for (auto &n : names) nvrtcAddNameExpression(prog, n.c_str());
  nvrtcResult rc = nvrtcCompileProgram(prog, nopts, opts);
  if (rc != NVRTC_SUCCESS) {
    size_t ls = 0;
    nvrtcGetProgramLogSize(prog, &ls);
    std::string l(ls, '\0');
    nvrtcGetProgramLog(prog, &l[0]);
    if (log) *log = std::string("NVRTC: ") + nvrtcGetErrorString(rc) + "\n" + l;
    nvrtcDestroyProgram(&prog);
    return false;
  }
  size_t cs = 0;
  nvrtcGetCUBINSize(prog, &cs);
  cubin->resize(cs);
  nvrtcGetCUBIN(prog, cubin->data());
  for (int i = 0; i < nk; ++i) {
    const char *ln = nullptr;
    nvrtcGetLoweredName(prog, names[i].c_str(), &ln);
    (*lowered)[i] = ln ? ln : "";
  }
  nvrtcDestroyProgram(&prog);
  // best-effort disk cache (atomic rename)
  mkdirs(dir);
  {
    std::ofstream fc(cubin_path + ".tmp", std::ios::binary);
    fc.write(cubin->data(), static_cast<std::streamsize>(cubin->size()));
  }
  {
    std::ofstream fn(names_path + ".tmp");
    for (auto &l : *lowered) fn << l << "\n";
  }
  std::rename((cubin_path + ".tmp").c_str(), cubin_path.c_str());
  std::rename((names_path + ".tmp").c_str(), names_path.c_str());
  return true;
}

bool device_is_sm100(std::string *log) {
  int dev = 0, major = 0, minor = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
  cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev);
  if (major != 10 || minor != 0) {
    if (log) *log = "runtime compilation targets sm_100a only";
    return false;
  }
  return true;
}

std::map<std::string, std::pair<cudaLibrary_t, AdjKernels>> g_adj_cache;

}  // namespace

bool jit_compile(const std::string &policy_source, bool fp32, std::vector<char> *cubin,
                 std::vector<std::string> *lowered, std::string *log) {
  const char *T = fp32 ? "float" : "double";
  const std::string src = "#include \"milne.cuh\"\nnamespace dl {\n" + policy_source + "}\n";
  const std::vector<std::string> names = {
      std::string("&dl::k_persistent<") + T + ", dl::YieldJit, false>",
      std::string("&dl::k_element<") + T + ", dl::YieldJit, false>",
      std::string("&dl::k_node<") + T + ", false>",
      std::string("&dl::k_internal_force<") + T + ", dl::YieldJit>",
      std::string("&dl::k_gather_force<") + T + ">",
      std::string("&dl::k_persistent<") + T + ", dl::YieldJit, true>",
      std::string("&dl::k_element<") + T + ", dl::YieldJit, true>",
      std::string("&dl::k_node<") + T + ", true>",
      std::string("&dl::k_milne<") + T + ", dl::YieldJit>",
      std::string("&dl::k_persistent<") + T + ", dl::YieldJit, false, true>"};
  return compile_generic(src, names, fp32, "step", cubin, lowered, log);
}

bool jit_compile_adjoint(const std::string &adj_policy_source, bool fp32, std::vector<char> *cubin,
                         std::vector<std::string> *lowered, std::string *log) {
  const char *T = fp32 ? "float" : "double";
  const std::string src = "#include \"adjoint_kernels.cuh\"\nnamespace dl {\n" + adj_policy_source + "}\n";
  const std::vector<std::string> names = {std::string("&dl::k_adj_node<") + T + ">",
                                          std::string("&dl::k_adj_elem<") + T + ", dl::YieldAdj>"};
  return compile_generic(src, names, fp32, "adjoint", cubin, lowered, log);
}

const AdjKernels *jit_adjoint_kernels(const std::string &adj_policy_source, bool fp32, std::string *log) {
  std::lock_guard<std::mutex> lock(g_mu);
  if (!device_is_sm100(log)) return nullptr;
  int dev = 0;
  cudaGetDevice(&dev);
  const std::string key = std::string(fp32 ? "f|" : "d|") + std::to_string(dev) + "|" + adj_policy_source;
  auto it = g_adj_cache.find(key);
  if (it != g_adj_cache.end()) return &it->second.second;
  std::vector<char> cubin;
  std::vector<std::string> lowered;
  if (!jit_compile_adjoint(adj_policy_source, fp32, &cubin, &lowered, log)) return nullptr;
  cudaLibrary_t lib = nullptr;
  if (cudaLibraryLoadData(&lib, cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0) != cudaSuccess) {
    cudaGetLastError();
    if (log) *log = "cudaLibraryLoadData failed";
    return nullptr;
  }
  cudaKernel_t k[2];
  for (int i = 0; i < 2; ++i)
    if (cudaLibraryGetKernel(&k[i], lib, lowered[i].c_str()) != cudaSuccess) {
      cudaGetLastError();
      if (log) *log = "cudaLibraryGetKernel failed for " + lowered[i];
      return nullptr;
    }
  AdjKernels ak;
  ak.node = reinterpret_cast<const void *>(k[0]);
  ak.elem = reinterpret_cast<const void *>(k[1]);
  auto &slot = g_adj_cache[key];
  slot = {lib, ak};
  return &slot.second;
}

const KernelSet *jit_kernels(const std::string &policy_source, bool fp32, std::string *log) {
  std::lock_guard<std::mutex> lock(g_mu);
  if (!device_is_sm100(log)) return nullptr;
  int dev = 0;
  cudaGetDevice(&dev);
  const std::string key = std::string(fp32 ? "f|" : "d|") + std::to_string(dev) + "|" + policy_source;
  auto it = g_cache.find(key);
  if (it != g_cache.end()) return &it->second->ks;
  std::vector<char> cubin;
  std::vector<std::string> lowered;
  if (!jit_compile(policy_source, fp32, &cubin, &lowered, log)) return nullptr;
  auto e = std::make_unique<Entry>();
  if (cudaLibraryLoadData(&e->lib, cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0) != cudaSuccess) {
    cudaGetLastError();
    if (log) *log = "cudaLibraryLoadData failed";
    return nullptr;
  }
  cudaKernel_t k[kNames];
  for (int i = 0; i < kNames; ++i)
    if (cudaLibraryGetKernel(&k[i], e->lib, lowered[i].c_str()) != cudaSuccess) {
      cudaGetLastError();
      if (log) *log = "cudaLibraryGetKernel failed for " + lowered[i];
      return nullptr;
    }
  e->ks.persistent = reinterpret_cast<const void *>(k[0]);
  e->ks.element = reinterpret_cast<const void *>(k[1]);
  e->ks.node = reinterpret_cast<const void *>(k[2]);
  e->ks.internal_force = reinterpret_cast<const void *>(k[3]);
  e->ks.gather = reinterpret_cast<const void *>(k[4]);
  e->ks.persistent_x = reinterpret_cast<const void *>(k[5]);
  e->ks.element_x = reinterpret_cast<const void *>(k[6]);
  e->ks.node_x = reinterpret_cast<const void *>(k[7]);
  e->ks.milne = reinterpret_cast<const void *>(k[8]);
  e->ks.persistent1 = reinterpret_cast<const void *>(k[9]);
  e->ks.full_threads = fp32 ? 320 : 256;  // PersistShape<T, false>::kThreads
  e->ks.full_threads_x = 256;             // PersistShape<T, true>::kThreads
  set_persistent_caps(e->ks);
  e->ks.jit = true;
  const KernelSet *out = &e->ks;
  g_cache[key] = std::move(e);
  return out;
}

}  // namespace dl
