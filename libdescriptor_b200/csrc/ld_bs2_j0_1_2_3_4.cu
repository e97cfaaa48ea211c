// ld_bs2_j0_1_2_3_4.cu -- instantiations of the twojmax-specialised bispectrum path.
#include "ld_bs2_impl.cuh"
namespace ldb {
template int bs2_launch_t<0>(const BSDev &, const RowArgs &, cudaStream_t);
template int bs2_launch_t<1>(const BSDev &, const RowArgs &, cudaStream_t);
template int bs2_launch_t<2>(const BSDev &, const RowArgs &, cudaStream_t);
template int bs2_launch_t<3>(const BSDev &, const RowArgs &, cudaStream_t);
template int bs2_launch_t<4>(const BSDev &, const RowArgs &, cudaStream_t);
}  // namespace ldb
