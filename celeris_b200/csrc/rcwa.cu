// RCWA entry points (filled in by the RCWA kernels).
#include "runtime.cuh"
extern "C" int celeris_solve_rcwa_2d(const celeris_rcwa_cell*, const double*, const double*, celeris_rcwa_result*) {
    return celeris_rt::set_error(CELERIS_ERR_INVALID_ARG, "RCWA not built yet");
}
extern "C" int celeris_rcwa_batch(const celeris_rcwa_cell*, int, celeris_rcwa_result*, int*) {
    return celeris_rt::set_error(CELERIS_ERR_INVALID_ARG, "RCWA not built yet");
}
