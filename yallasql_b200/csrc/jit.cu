// Program-specialised row kernels, compiled at run time for sm_100a.
//
// The row kernels (row_kernels.cuh) are templates over a program runner. The
// library's own kernels use the interpreter runner, which dispatches on each
// resolved opcode at run time. For a program seen by the library, this file
// writes a small CUDA source whose runner lists the program's instructions as
// compile-time constants - `exec<opcode>(P, {opcode, flags, operands}, ...)`
// one after another - so the same operation bodies compile to straight-line
// code with the opcode dispatch and the stack moves folded away. NVRTC (opened
// with dlopen; nothing links against it) compiles that source together with
// the library's device headers, embedded at build time, straight to an
// sm_100a cubin; the cubin is loaded with cudaLibraryLoadData and launched
// with cudaLaunchKernel. Kernels are cached per (kind, staging, instruction
// words): constants are kernel parameters, so a program that differs only in
// its constants reuses the kernel.
//
// Switched off by YQ_JIT=0 in the environment or yq_jit_enable(0); any
// failure (no NVRTC, a compile error) leaves the interpreter kernels in use.
#include <dlfcn.h>
#include <chrono>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <array>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>
#include <nvrtc.h>  // types and prototypes only
#include "yq_jit.cuh"
#include "row_kernels.cuh"

// Device headers embedded by the build (yallasql_b200/build.py).
extern const int yq_jit_header_count;
extern const char* const yq_jit_header_names[];
extern const char* const yq_jit_header_texts[];

namespace yq {

namespace {

struct Nvrtc {
  decltype(&nvrtcCreateProgram) create = nullptr;
  decltype(&nvrtcCompileProgram) compile = nullptr;
  decltype(&nvrtcGetProgramLogSize) log_size = nullptr;
  decltype(&nvrtcGetProgramLog) log = nullptr;
  decltype(&nvrtcGetCUBINSize) cubin_size = nullptr;
  decltype(&nvrtcGetCUBIN) cubin = nullptr;
  decltype(&nvrtcDestroyProgram) destroy = nullptr;
  bool ok = false;
};

std::mutex g_mu;
int g_enabled = -1;  // -1: not decided yet (environment)
Nvrtc g_nvrtc;
bool g_nvrtc_tried = false;
std::unordered_map<std::string, const void*> g_cache;  // null entries: compile failed
int g_compiled = 0, g_failed = 0, g_hits = 0;
double g_compile_ms = 0;
std::string g_last_log;
std::vector<std::vector<char>> g_images;  // cubins of the loaded libraries, kept for the process

bool open_nvrtc() {
  if (g_nvrtc_tried) return g_nvrtc.ok;
  g_nvrtc_tried = true;
  const char* names[] = {"libnvrtc.so.12", "libnvrtc.so", "/usr/local/cuda/lib64/libnvrtc.so.12"};
  void* h = nullptr;
  for (const char* n : names)
    if ((h = dlopen(n, RTLD_NOW | RTLD_LOCAL))) break;
  if (!h) {
    g_last_log = "libnvrtc not found";
    return false;
  }
  g_nvrtc.create = reinterpret_cast<decltype(g_nvrtc.create)>(dlsym(h, "nvrtcCreateProgram"));
  g_nvrtc.compile = reinterpret_cast<decltype(g_nvrtc.compile)>(dlsym(h, "nvrtcCompileProgram"));
  g_nvrtc.log_size = reinterpret_cast<decltype(g_nvrtc.log_size)>(dlsym(h, "nvrtcGetProgramLogSize"));
  g_nvrtc.log = reinterpret_cast<decltype(g_nvrtc.log)>(dlsym(h, "nvrtcGetProgramLog"));
  g_nvrtc.cubin_size = reinterpret_cast<decltype(g_nvrtc.cubin_size)>(dlsym(h, "nvrtcGetCUBINSize"));
  g_nvrtc.cubin = reinterpret_cast<decltype(g_nvrtc.cubin)>(dlsym(h, "nvrtcGetCUBIN"));
  g_nvrtc.destroy = reinterpret_cast<decltype(g_nvrtc.destroy)>(dlsym(h, "nvrtcDestroyProgram"));
  g_nvrtc.ok = g_nvrtc.create && g_nvrtc.compile && g_nvrtc.log_size && g_nvrtc.log && g_nvrtc.cubin_size &&
               g_nvrtc.cubin && g_nvrtc.destroy;
  if (!g_nvrtc.ok) g_last_log = "libnvrtc lacks an entry point";
  return g_nvrtc.ok;
}

bool enabled_locked() {
  if (g_enabled < 0) {
    const char* e = getenv("YQ_JIT");
    g_enabled = (e && e[0] == '0') ? 0 : 1;
  }
  return g_enabled == 1;
}

const char* kernel_decl(JitKind kind) {
  switch (kind) {
    case JIT_FILTER_AGG:
      return "(const __grid_constant__ yq::FAParams F, uint32_t n, yq::Acc* __restrict__ partials, uint32_t* ticket,"
             " yq::Acc* state) { yq::filter_aggregate_body<STAGED_, yq::JitRunner>(F, n, partials, ticket, state); }";
    case JIT_FILTER_AGG_SEG:
      return "(const __grid_constant__ yq::FASegParams Q) { yq::filter_aggregate_seg_body<STAGED_, yq::JitRunner>(Q); }";
    case JIT_FILTER_PROJECT:
      return "(const __grid_constant__ yq::FPParams F, uint32_t n, uint32_t* tile_counter,"
             " unsigned long long* __restrict__ status, uint32_t* out_count, uint32_t* err) {"
             " yq::filter_project_body<STAGED_, yq::JitRunner>(F, n, tile_counter, status, out_count, err); }";
    default:
      return "(const __grid_constant__ yq::JAParams F, uint32_t n, yq::Acc* __restrict__ partials, uint32_t* ticket,"
             " yq::Acc* state) { yq::join_aggregate_body<STAGED_, yq::JitRunner>(F, n, partials, ticket, state); }";
  }
}

// The source-column copies of a WHERE + projection: (output, column, width,
// output nulls, source nulls) for each projection that copies a column.
std::vector<std::array<int, 5>> copy_list(const FPParams* fp) {
  std::vector<std::array<int, 5>> v;
  if (!fp) return v;
  for (int p = 0; p < fp->nproj; ++p) {
    const DevOut& o = fp->out[p];
    if (o.src_col < 0) continue;
    v.push_back({p, o.src_col, o.width, o.nulls ? 1 : 0, fp->P.cols[o.src_col].nulls ? 1 : 0});
  }
  return v;
}

std::string make_source(JitKind kind, bool staged, const VmProgram& P, int seg0_end, int end, int min_blocks,
                        const FPParams* fp) {
  std::string s;
  s += "#include \"row_kernels.cuh\"\n#define STAGED_ ";
  s += staged ? "true" : "false";
  s += "\nnamespace yq {\nstruct JitRunner {\n  template <bool STAGED, typename Emit>\n"
       "  __device__ __forceinline__ static void run(const VmProgram& P, int seg, int, int, const Ctx& X, Stack& S,"
       " Emit& E) {\n";
  char line[256];
  for (int seg = 0; seg < 2; ++seg) {
    const int b = seg == 0 ? 0 : seg0_end, e = seg == 0 ? seg0_end : end;
    s += seg == 0 ? "    if (seg == 0) {\n" : "    } else {\n";
    for (int i = b; i < e; ++i) {
      const RInsn& I = P.code[i];
      snprintf(line, sizeof(line),
               "      { constexpr RInsn I{%u, %u, %u, %u, %u, %u}; exec<%u, STAGED>(P, I, X, S, E); }\n",
               (unsigned)I.opc, (unsigned)I.flags, (unsigned)I.a, (unsigned)I.b, (unsigned)I.c, (unsigned)I.imm,
               (unsigned)I.opc);
      s += line;
    }
  }
  s += "    }\n  }\n";
  if (kind == JIT_FILTER_PROJECT) {
    s += "  template <bool STAGED>\n  __device__ __forceinline__ static void copies(const FPParams& F, const Ctx& X,"
         " const ProjEmit& E) {\n";
    for (const auto& c : copy_list(fp)) {
      snprintf(line, sizeof(line), "    copy_column<STAGED, %d, %d, %d, %s, %s>(F, X, E);\n", c[0], c[1], c[2],
               c[3] ? "true" : "false", c[4] ? "true" : "false");
      s += line;
    }
    s += "  }\n";
  }
  s += "};\n}  // namespace yq\n";
  s += "extern \"C\" __global__ void __launch_bounds__(256, " + std::to_string(min_blocks) + ") yq_jit_kernel";
  s += kernel_decl(kind);
  s += "\n";
  return s;
}

std::string cache_key(JitKind kind, bool staged, const VmProgram& P, int seg0_end, int end, const FPParams* fp) {
  std::string k;
  k.reserve(16 + (size_t)end * sizeof(RInsn));
  k += (char)('0' + (int)kind);
  k += staged ? 'S' : 'G';
  k.append(reinterpret_cast<const char*>(&seg0_end), sizeof(int));
  k.append(reinterpret_cast<const char*>(&end), sizeof(int));
  k.append(reinterpret_cast<const char*>(P.code), (size_t)end * sizeof(RInsn));
  if (kind == JIT_FILTER_PROJECT)
    for (const auto& c : copy_list(fp)) k.append(reinterpret_cast<const char*>(c.data()), sizeof(int) * 5);
  return k;
}

// Spill stores ptxas reported for the kernel entry (-1 when not found).
long entry_spills(const std::string& log) {
  const size_t at = log.find("Function properties for yq_jit_kernel");
  if (at == std::string::npos) return -1;
  const size_t sp = log.find("bytes spill stores", at);
  if (sp == std::string::npos) return -1;
  const size_t b = log.rfind(',', sp);  // "N bytes stack frame, N bytes spill stores"
  if (b == std::string::npos || b < at) return -1;
  return strtol(log.c_str() + b + 1, nullptr, 10);
}

// Compiles and loads one kernel source. `spills` receives the entry's spill
// stores as ptxas reported them.
const void* compile_locked(const std::string& src, long* spills) {
  nvrtcProgram prog = nullptr;
  if (g_nvrtc.create(&prog, src.c_str(), "yq_jit.cu", yq_jit_header_count, yq_jit_header_texts,
                     yq_jit_header_names) != NVRTC_SUCCESS) {
    g_last_log = "nvrtcCreateProgram failed";
    return nullptr;
  }
  // -default-device: the C declarations of the public header are never defined
  // or called here; 9 = nested comment in the header's prose.
  const char* opts[] = {"-arch=sm_100a", "-std=c++17", "-DNDEBUG", "-default-device", "-diag-suppress=9",
                        "--ptxas-options=-v"};
  const nvrtcResult r = g_nvrtc.compile(prog, 6, opts);
  size_t ls = 0;
  g_nvrtc.log_size(prog, &ls);
  std::string log(ls, '\0');
  if (ls) g_nvrtc.log(prog, &log[0]);
  g_last_log = log;
  *spills = entry_spills(log);
  const void* kernel = nullptr;
  if (r == NVRTC_SUCCESS) {
    size_t n = 0;
    g_nvrtc.cubin_size(prog, &n);
    std::vector<char> cubin(n);
    if (n && g_nvrtc.cubin(prog, cubin.data()) == NVRTC_SUCCESS) {
      cudaLibrary_t lib = nullptr;
      cudaKernel_t k = nullptr;
      g_images.push_back(std::move(cubin));
      if (cudaLibraryLoadData(&lib, g_images.back().data(), nullptr, nullptr, 0, nullptr, nullptr, 0) == cudaSuccess &&
          cudaLibraryGetKernel(&k, lib, "yq_jit_kernel") == cudaSuccess)
        kernel = reinterpret_cast<const void*>(k);  // the library stays loaded for the process
      else
        g_last_log += "\ncubin load failed";
      cudaGetLastError();
    }
  }
  g_nvrtc.destroy(&prog);
  return kernel;
}

}  // namespace

const void* jit_kernel(JitKind kind, bool staged, const VmProgram& P, int seg0_end, int end, const FPParams* fp) {
  if (end < 0 || end > kMaxInsns || seg0_end < 0 || seg0_end > end) return nullptr;
  std::lock_guard<std::mutex> lk(g_mu);
  if (!enabled_locked()) return nullptr;
  const std::string key = cache_key(kind, staged, P, seg0_end, end, fp);
  auto it = g_cache.find(key);
  if (it != g_cache.end()) {
    ++g_hits;
    return it->second;
  }
  const void* k = nullptr;
  if (open_nvrtc()) {
    const auto t0 = std::chrono::steady_clock::now();
    // Registers for four blocks of 256 threads per SM (64 a thread) when the
    // kernel fits them without spilling, else for three, else for two.
    long spills = 0;
    for (int blocks = 4; blocks >= 2; --blocks) {
      k = compile_locked(make_source(kind, staged, P, seg0_end, end, blocks, fp), &spills);
      if (!k || spills == 0) break;
    }
    g_compile_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  }
  if (k) ++g_compiled;
  else ++g_failed;
  g_cache.emplace(key, k);
  return k;
}

namespace {

std::mutex g_launch_mu;
std::unordered_map<std::string, size_t> g_smem_cap;  // dynamic shared memory a kernel allows, per device
std::unordered_map<std::string, int> g_resident;     // blocks per SM per (kernel, shared memory, device)
std::unordered_map<std::string, int> g_depth;        // ring depth per (kernel, stage bytes, device)

std::string launch_key(const void* kernel, size_t extra, int dev) {
  std::string k(reinterpret_cast<const char*>(&kernel), sizeof(kernel));
  k.append(reinterpret_cast<const char*>(&extra), sizeof(extra));
  k.append(reinterpret_cast<const char*>(&dev), sizeof(dev));
  return k;
}

// Lets `kernel` take `smem` bytes of dynamic shared memory on `dev`. The cap
// only ever rises, so a launch with less never lowers what another needs.
cudaError_t allow_smem_locked(const void* kernel, size_t smem, int dev) {
  if (smem <= 48 * 1024) return cudaSuccess;
  size_t& cap = g_smem_cap[launch_key(kernel, 0, dev)];
  if (smem <= cap) return cudaSuccess;
  cudaKernel_t k = reinterpret_cast<cudaKernel_t>(const_cast<void*>(kernel));
  const cudaError_t e = cudaKernelSetAttributeForDevice(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem, dev);
  if (e == cudaSuccess) cap = smem;
  return e;
}

// Blocks of 256 threads per SM (0 when the shared memory cannot be allowed).
int resident_locked(const void* kernel, size_t smem, int dev) {
  const std::string key = launch_key(kernel, smem, dev);
  auto it = g_resident.find(key);
  if (it != g_resident.end()) return it->second;
  int per_sm = 0;
  if (allow_smem_locked(kernel, smem, dev) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 256, smem) != cudaSuccess)
    per_sm = 0;
  cudaGetLastError();
  g_resident.emplace(key, per_sm);
  return per_sm;
}

}  // namespace

int jit_stages(const void* kernel, uint32_t stage_bytes, int nstages, size_t extra) {
  if (!kernel || nstages < 2 || stage_bytes == 0) return nstages;
  static int fit = -1;
  std::lock_guard<std::mutex> lk(g_launch_mu);
  if (fit < 0) {
    const char* e = getenv("YQ_STAGE_FIT");
    fit = (e && e[0] == '0') ? 0 : 1;
  }
  if (!fit) return nstages;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return nstages;
  }
  const std::string key = launch_key(kernel, stage_bytes, dev) + std::string(reinterpret_cast<const char*>(&extra),
                                                                          sizeof(extra));
  auto it = g_depth.find(key);
  if (it != g_depth.end()) return it->second;
  int best = nstages, best_blocks = 0;
  for (int ns = 2; ns <= kStageMax; ++ns) {  // deeper on a tie
    const size_t ring = (size_t)ns * stage_bytes + (size_t)ns * 8;
    const int per_sm = resident_locked(kernel, extra ? align_up(ring, 16) + extra : ring, dev);
    if (per_sm == 0) break;
    if (per_sm >= best_blocks) {
      best_blocks = per_sm;
      best = ns;
    }
  }
  g_depth.emplace(key, best);
  return best;
}

int jit_launch(const void* kernel, int max_grid, uint32_t steps, size_t smem, void** args, cudaStream_t s) {
  int dev = 0;
  YQ_TRY_CUDA(cudaGetDevice(&dev));
  int per_sm = 0;
  {
    std::lock_guard<std::mutex> lk(g_launch_mu);
    per_sm = resident_locked(kernel, smem, dev);
    if (per_sm == 0) {  // shared memory not allowed: report it
      const cudaError_t e = allow_smem_locked(kernel, smem, dev);
      set_cuda_error(e == cudaSuccess ? cudaErrorInvalidConfiguration : e);
      return YQ_ERR_CUDA;
    }
  }
  int grid = per_sm * sm_count();
  if (grid > max_grid) grid = max_grid;
  if ((uint32_t)grid > steps) grid = (int)steps;
  if (grid < 1) grid = 1;
  YQ_TRY_CUDA(cudaLaunchKernel(kernel, dim3((unsigned)grid), dim3(256), args, smem, s));
  count_launch();
  return YQ_OK;
}

}  // namespace yq

extern "C" {

int yq_jit_enable(int32_t on) {
  std::lock_guard<std::mutex> lk(yq::g_mu);
  const int before = yq::enabled_locked() ? 1 : 0;
  yq::g_enabled = on ? 1 : 0;
  return before;
}

int yq_jit_stats(int32_t* compiled, int32_t* failed, int32_t* hits, double* compile_ms, char* log, size_t log_bytes) {
  std::lock_guard<std::mutex> lk(yq::g_mu);
  if (compiled) *compiled = yq::g_compiled;
  if (failed) *failed = yq::g_failed;
  if (hits) *hits = yq::g_hits;
  if (compile_ms) *compile_ms = yq::g_compile_ms;
  if (log && log_bytes) {
    const size_t n = yq::g_last_log.size() < log_bytes - 1 ? yq::g_last_log.size() : log_bytes - 1;
    memcpy(log, yq::g_last_log.data(), n);
    log[n] = '\0';
  }
  return YQ_OK;
}

}  // extern "C"
