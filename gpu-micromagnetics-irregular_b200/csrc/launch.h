// launch.h — kernel launches with programmatic dependent launch (PDL).
//
// Kernels of the integrator's hot loop are launched with the
// programmatic-stream-serialisation attribute and begin with pdl_entry():
// griddepcontrol.wait holds this kernel until the previous one has finished
// and its memory is visible, then griddepcontrol.launch_dependents lets the
// next kernel of the stream be scheduled.  The next launch's set-up therefore
// overlaps the body of the current kernel instead of following it.  Both
// instructions are no-ops for a kernel launched without the attribute.
//
// The order matters.  Triggering before waiting lets kernel C (after B after
// A) be dispatched while A still runs; C's SMs may then keep lines that A
// loaded, and when B rewrites them in place (the Gram-Schmidt update of a
// Krylov vector between its dot products and its normalisation) C reads the
// old values through the non-coherent load path that const __restrict__
// pointers compile to.  Waiting first means a kernel is dispatched only after
// every kernel two places before it in the stream has finished.
//
// A PDL launch relaxes the dependency on the preceding kernel only, so it is
// used only where every operation of the stream between two such kernels is
// itself a kernel: inside the host integrator's step loop on the legacy
// default stream (PdlScope).  Elsewhere — graph capture, streams that replay
// the demag chain as a graph, set-up copies — g_no_pdl keeps launches plain.


#pragma once
#include <cuda_runtime.h>

extern thread_local int g_no_pdl;
extern thread_local int g_pdl_break;   // the next launch follows a non-kernel operation: plain

// The first launch of a scope follows whatever the caller left on the stream,
// so it is plain too.
struct PdlScope {
  int saved;
  explicit PdlScope(bool on) : saved(g_no_pdl) {
    if (on) g_no_pdl = 0;
    g_pdl_break = 1;
  }
  ~PdlScope() { g_no_pdl = saved; }
};
inline void pdl_break() { g_pdl_break = 1; }

template <typename... KArgs, typename... Args>
inline void klaunch(void (*kernel)(KArgs...), dim3 g, dim3 b, size_t smem, cudaStream_t s, Args... args) {
#ifdef LLG_PLAIN_LAUNCH
  if (true) {
#else
  if (g_no_pdl || g_pdl_break) {
#endif
    g_pdl_break = 0;
    kernel<<<g, b, smem, s>>>(args...);
    return;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = g;
  cfg.blockDim = b;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  (void)cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

#ifdef __CUDACC__
__device__ __forceinline__ void pdl_entry() {
  asm volatile("griddepcontrol.wait;\n" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
}
#endif
