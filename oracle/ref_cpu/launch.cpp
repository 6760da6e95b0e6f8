// CPU launchers for the reference kernels (kernels.cu, compiled unmodified
// as C++ with shim/cuda_cpu.h force-included).  Each launcher walks the
// launch grid serially, setting blockIdx/threadIdx before every call, so the
// kernel bodies run exactly as written, one thread at a time.
//
// Test infrastructure only: used by tests/golden/make_golden.py (through the
// NumPy stand-in for cupy.RawModule) to run the reference's own emc.py /
// maxLP.py code on the CPU.  Built by oracle/ref_cpu/build.py into
// oracle/_ref/.
#include "kernels.cu"

thread_local rspi_cpu_dim3 threadIdx, blockIdx, blockDim, gridDim;

template <class F>
static void run_grid(unsigned gx, unsigned gy, unsigned bx, unsigned by, F f) {
    gridDim = {gx, gy, 1};
    blockDim = {bx, by, 1};
    for (unsigned j = 0; j < gy; ++j)
        for (unsigned i = 0; i < gx; ++i)
            for (unsigned ty = 0; ty < by; ++ty)
                for (unsigned tx = 0; tx < bx; ++tx) {
                    blockIdx = {i, j, 0};
                    threadIdx = {tx, ty, 0};
                    f();
                }
}

extern "C" {

void ref_slice_gen(unsigned gx, unsigned gy, unsigned bx, unsigned by,
                   const double *model, double angle, double scale, long long size,
                   const double *bg, long long log_flag, double *view) {
    run_grid(gx, gy, bx, by, [&] { slice_gen(model, angle, scale, size, bg, log_flag, view); });
}

void ref_slice_gen_holo(unsigned gx, unsigned gy, unsigned bx, unsigned by,
                        const complex<double> *model, double shiftx, double shifty,
                        double diameter, double rel_scale, double scale, long long size,
                        const double *bg, long long log_flag, double *view) {
    run_grid(gx, gy, bx, by, [&] {
        slice_gen_holo(model, shiftx, shifty, diameter, rel_scale, scale, size, bg, log_flag, view);
    });
}

void ref_slice_merge(unsigned gx, unsigned gy, unsigned bx, unsigned by,
                     const double *view, double angle, long long size,
                     double *model, double *mweights) {
    run_grid(gx, gy, bx, by, [&] { slice_merge(view, angle, size, model, mweights); });
}

void ref_calc_prob_all(unsigned gx, unsigned bx, const double *lview, const int *mask,
                       long long ndata, const int *ones, const int *multi,
                       const long long *o_acc, const long long *m_acc, const int *p_o,
                       const int *p_m, const int *c_m, double init, const double *scales,
                       double *prob_r) {
    run_grid(gx, 1, bx, 1, [&] {
        calc_prob_all(lview, mask, ndata, ones, multi, o_acc, m_acc, p_o, p_m, c_m, init,
                      scales, prob_r);
    });
}

void ref_merge_all(unsigned gx, unsigned bx, const double *prob_r, long long ndata,
                   const int *ones, const int *multi, const long long *o_acc,
                   const long long *m_acc, const int *p_o, const int *p_m, const int *c_m,
                   double *view) {
    run_grid(gx, 1, bx, 1, [&] {
        merge_all(prob_r, ndata, ones, multi, o_acc, m_acc, p_o, p_m, c_m, view);
    });
}

void ref_get_f_dt(unsigned gx, unsigned bx, const complex<double> *fobj_t,
                  const complex<double> *fref_d, long long ndata, long long npix,
                  complex<double> *f_dt) {
    run_grid(gx, 1, bx, 1, [&] { get_f_dt(fobj_t, fref_d, ndata, npix, f_dt); });
}

}  // extern "C"
