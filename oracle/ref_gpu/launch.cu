// GPU launchers for the reference kernels (kernels.cu, compiled unmodified
// by nvcc with shim/ standing in for <cupy/complex.cuh>).  Each launcher
// takes the grid and block the reference's emc.py / maxLP.py pass to the
// CuPy RawModule kernel and the CUDA stream to launch on, so a Python
// replay of the reference's loops runs the reference's own device code on
// the same GPU.
//
// Test and baseline infrastructure only (oracle/): used by the GPU tests
// that compare the product against the reference's kernels and by the
// reference arm of bench.py.  Built by oracle/ref_gpu/build.py into
// oracle/_ref/.
#include "kernels.cu"

extern "C" {

int ref_gpu_slice_gen(unsigned gx, unsigned gy, unsigned bx, unsigned by, const double *model,
                      double angle, double scale, long long size, const double *bg,
                      long long log_flag, double *view, cudaStream_t stream) {
    slice_gen<<<dim3(gx, gy), dim3(bx, by), 0, stream>>>(model, angle, scale, size, bg, log_flag,
                                                         view);
    return (int)cudaGetLastError();
}

int ref_gpu_slice_gen_holo(unsigned gx, unsigned gy, unsigned bx, unsigned by,
                           const complex<double> *model, double shiftx, double shifty,
                           double diameter, double rel_scale, double scale, long long size,
                           const double *bg, long long log_flag, double *view,
                           cudaStream_t stream) {
    slice_gen_holo<<<dim3(gx, gy), dim3(bx, by), 0, stream>>>(
        model, shiftx, shifty, diameter, rel_scale, scale, size, bg, log_flag, view);
    return (int)cudaGetLastError();
}

int ref_gpu_calc_prob_all(unsigned gx, unsigned bx, const double *lview, const int *mask,
                          long long ndata, const int *ones, const int *multi,
                          const long long *o_acc, const long long *m_acc, const int *p_o,
                          const int *p_m, const int *c_m, double init, const double *scales,
                          double *prob_r, cudaStream_t stream) {
    calc_prob_all<<<gx, bx, 0, stream>>>(lview, mask, ndata, ones, multi, o_acc, m_acc, p_o, p_m,
                                         c_m, init, scales, prob_r);
    return (int)cudaGetLastError();
}

int ref_gpu_get_f_dt(unsigned gx, unsigned bx, const complex<double> *fobj_t,
                     const complex<double> *fref_d, long long ndata, long long npix,
                     complex<double> *f_dt, cudaStream_t stream) {
    get_f_dt<<<gx, bx, 0, stream>>>(fobj_t, fref_d, ndata, npix, f_dt);
    return (int)cudaGetLastError();
}

}  // extern "C"
