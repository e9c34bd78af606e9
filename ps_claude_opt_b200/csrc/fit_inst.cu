// fit_inst.cu -- one instance of the fit kernel, compiled once per padded
// coefficient count (-DPSB_NCP=16..88), precision (-DPSB_MIXED=0/1) and
// form (-DPSB_BATCH=1: many objects per launch) so the instances build in
// parallel.
#include "fit_kernel.cuh"

#ifndef PSB_NCP
#error "compile with -DPSB_NCP=<padded coefficient count>"
#endif
#ifndef PSB_MIXED
#define PSB_MIXED 0
#endif
#ifndef PSB_BATCH
#define PSB_BATCH 0
#endif

namespace psb {

using KernelFn = void (*)(DevObject, DevParams, const FitItem *, int, int *, FitOut *, double *, size_t,
                          int *, EvalOut, int, const DevObject *, const DevParams *);

#define PSB_CAT2(a, b) a##b
#define PSB_CAT(a, b) PSB_CAT2(a, b)
#if PSB_BATCH
KernelFn PSB_CAT(fit_kernel_batch_ptr_, PSB_NCP)() { return fit_kernel<PSB_NCP, false, true>; }
#elif PSB_MIXED
KernelFn PSB_CAT(fit_kernel_mixed_ptr_, PSB_NCP)() { return fit_kernel<PSB_NCP, true, false>; }
#else
KernelFn PSB_CAT(fit_kernel_ptr_, PSB_NCP)() { return fit_kernel<PSB_NCP, false, false>; }
#endif

}  // namespace psb
