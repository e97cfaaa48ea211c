// ld_bs2_j8.cu -- instantiations of the twojmax-specialised bispectrum path.
#include "ld_bs2_impl.cuh"
namespace ldb {
template int bs2_launch_t<8>(const BSDev &, const RowArgs &, cudaStream_t);
}  // namespace ldb
