// ld_bs2_j5_6.cu -- instantiations of the twojmax-specialised bispectrum path.
#include "ld_bs2_impl.cuh"
namespace ldb {
template int bs2_launch_t<5>(const BSDev &, const RowArgs &, cudaStream_t);
template int bs2_launch_t<6>(const BSDev &, const RowArgs &, cudaStream_t);
}  // namespace ldb
