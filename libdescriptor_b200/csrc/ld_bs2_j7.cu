// ld_bs2_j7.cu -- instantiations of the twojmax-specialised bispectrum path.
#include "ld_bs2_impl.cuh"
namespace ldb {
template int bs2_launch_t<7>(const BSDev &, const RowArgs &, cudaStream_t);
}  // namespace ldb
