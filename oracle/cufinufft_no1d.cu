// Link stand-ins for the 1D spreader of the reference's vendored cuFINUFFT
// (external/finufft/src/cuda/1d/spread1d_wrapper.cu), whose compilation for
// sm_100a crashes the CUDA 12.9 device front end (cicc segmentation fault).
// The benchmark's reference bar only makes 3D type-1 plans, so the 1D spread
// entry points that cufinufft.cu's dimension dispatch names answer
// FINUFFT_ERR_DIM_NOTVALID.  Test and baseline infrastructure only.
#include <cufinufft/spreadinterp.h>
#include <cufinufft/types.h>
#include <finufft_errors.h>

namespace cufinufft {
namespace spreadinterp {

template<typename T> int cuspread1d(cufinufft_plan_t<T> *, int) {
  return FINUFFT_ERR_DIM_NOTVALID;
}
template<typename T> int cuspread1d_nuptsdriven_prop(int, int, cufinufft_plan_t<T> *) {
  return FINUFFT_ERR_DIM_NOTVALID;
}
template<typename T> int cuspread1d_subprob_prop(int, int, cufinufft_plan_t<T> *) {
  return FINUFFT_ERR_DIM_NOTVALID;
}

template int cuspread1d<float>(cufinufft_plan_t<float> *, int);
template int cuspread1d<double>(cufinufft_plan_t<double> *, int);
template int cuspread1d_nuptsdriven_prop<float>(int, int, cufinufft_plan_t<float> *);
template int cuspread1d_nuptsdriven_prop<double>(int, int, cufinufft_plan_t<double> *);
template int cuspread1d_subprob_prop<float>(int, int, cufinufft_plan_t<float> *);
template int cuspread1d_subprob_prop<double>(int, int, cufinufft_plan_t<double> *);

}  // namespace spreadinterp
}  // namespace cufinufft
