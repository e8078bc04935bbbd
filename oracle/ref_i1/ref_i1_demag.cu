// ref_i1_demag.cu — the reference's periodic cuFFT demag module of the 2d_i1
// variant (Demag_Init / Demag_Apply / Demag_GetSelfCoupling / Demag_Destroy),
// compiled from src/irregular/2d_fft/2d_i1/demag_fft.cu where it lies, for the
// RHS wrapper f of ref_i1_f.cu.  TEST INFRASTRUCTURE ONLY.
#include "demag_fft.cu"
