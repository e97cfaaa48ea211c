// Descriptors.hpp -- C++ drop-in for libdescriptor's driver API, served by the
// B200 library (link libldb200_cxx.so, which sits on the C ABI of
// include/libdescriptor_b200.h).
//
// Put this directory on the include path in place of the reference's
// include/ and a call site written against the reference's header
// (include/Descriptors.hpp:19-271: namespace Descriptor, its free functions
// and class DescriptorKind with the initDescriptor overloads) compiles and
// links unchanged.  The declarations keep the reference's names, argument
// lists and meanings; the code behind them is this library's.
//
// Semantics kept from the reference:
//  * compute / compute_batch / gradient* add symmetry-function descriptors
//    into desc (the caller zeroes it) and overwrite bispectrum descriptors;
//  * the gradients and the Jacobian are ADDED into d_coordinates /
//    J_coordinates (the caller zeroes them), rows of all coordinates
//    (contributing atoms and ghosts), unfolded;
//  * errors throw std::invalid_argument (bad arguments, unsupported kinds)
//    or std::runtime_error (device failures).
// Differences: dE_dzeta is never modified (the reference's Enzyme pass may
// zero it); descriptor_kind is set by every initDescriptor overload (the
// reference's symmetry-function overload leaves it unset); the number of
// coordinate rows, which the reference never needs, is taken as one past the
// largest centre or neighbour index; SOAP and Xi are not provided (their
// overloads throw).
#ifndef LIBDESCRIPTOR_B200_CXX_DESCRIPTORS_HPP_
#define LIBDESCRIPTOR_B200_CXX_DESCRIPTORS_HPP_

#include <stdexcept>
#include <string>
#include <vector>

namespace Descriptor {

// numbered as the reference's enum (include/Descriptors.hpp:21-26)
enum AvailableDescriptor { KindSymmetryFunctions, KindBispectrum, KindSOAP, KindXi };

class DescriptorKind;

// forward-mode differentiation is not implemented by the reference either
inline void fwd_diff(int, int *, int *, int *, double *, double *, DescriptorKind *) {
    throw std::logic_error("Function not implemented yet.");
}

// d_coordinates += dE_dzeta . d desc / d coordinates over all contributing atoms
void gradient(int n_atoms, int *species, int *neighbor_list, int *number_of_neighs, double *coordinates,
              double *d_coordinates, double *desc, double *dE_dzeta, DescriptorKind *descriptor_to_diff);

// the same over a batch: centre of row (c, j) is j + config_ptr[c]
void gradient_batch(int n_configurations, int *n_atoms, int *config_ptr, int *species, int *neighbor_list,
                    int *number_of_neighs, double *coordinates, double *d_coordinates, double *desc,
                    double *dE_dzeta, DescriptorKind *descriptor_to_diff);

// the same for the one centre `index` with its own neighbour list
void gradient_single_atom(int index, int n_atoms, int *species, int *neighbor_list, int number_of_neighs,
                          double *coordinates, double *d_coordinates, double *desc, double *dE_dzeta,
                          DescriptorKind *descriptor_to_diff);

// d_coordinates[0..2] += dE_dzeta . d desc_index / d x_index by the
// reference's 8th-order central finite difference
void num_gradient_single_atom(int index, int n_atoms, int *species, int *neighbor_list, int number_of_neighs,
                              double *coordinates, double *d_coordinates, double *dE_dzeta,
                              DescriptorKind *descriptor_to_diff);

// J_coordinates[(width n_atoms) x (3 n_total_atoms)] += d desc_flat / d coordinates_flat
void jacobian(int n_atoms, int n_total_atoms, int *species, int *neighbor_list, int *number_of_neighs,
              double *coordinates, double *J_coordinates, DescriptorKind *descriptor_to_diff);

// descriptors of the contributing atoms 0 .. n_atoms-1, rows in order
void compute(int n_atoms, int *species, int *neighbor_list, int *number_of_neighs, double *coordinates,
             double *desc, DescriptorKind *descriptor_kind);

void compute_batch(int n_configurations, int *n_atoms, int *config_ptr, int *species, int *neighbor_list,
                   int *number_of_neighs, double *coordinates, double *desc, DescriptorKind *descriptor_kind);

void compute_single_atom(int index, int n_atoms, int *species, int *neighbor_list, int number_of_neighs,
                         double *coordinates, double *desc, DescriptorKind *descriptor_kind);

}  // namespace Descriptor

// Base class of the descriptor kinds.  The initDescriptor overloads return
// kinds served by the B200 library; a caller's own subclass keeps working
// with compute / compute_batch / compute_single_atom (its virtual compute is
// called per centre), while the gradients need a library kind.
class Descriptor::DescriptorKind {
   public:
    AvailableDescriptor descriptor_kind;  // kind of this descriptor
    std::string descriptor_param_file;    // parameter file it was read from, if any
    int width = -1;                       // descriptor dimension

    DescriptorKind() = default;

    // an empty kind (no parameters): its compute throws
    static DescriptorKind *initDescriptor(AvailableDescriptor availableDescriptorKind);

    // from a parameter file in the reference's format
    static DescriptorKind *initDescriptor(std::string &file_name, AvailableDescriptor availableDescriptorKind);

    // descriptor of centre `index` into desc[width]
    virtual void compute(int index, int n_atoms, int *species, int *neighbor_lists, int number_of_neighbors,
                         double *coordinates, double *desc) = 0;

    virtual ~DescriptorKind();

    // symmetry functions: cutoff[0] for every species pair
    static DescriptorKind *initDescriptor(AvailableDescriptor availableDescriptorKind,
                                          std::vector<std::string> *species, std::string *cutoff_function,
                                          double *cutoff_matrix, std::vector<std::string> *symmetry_function_types,
                                          std::vector<int> *symmetry_function_sizes,
                                          std::vector<double> *symmetry_function_parameters);

    // bispectrum: cutoff_array[0] for every species pair
    static DescriptorKind *initDescriptor(AvailableDescriptor availableDescriptorKind, double rfac0_in,
                                          int twojmax_in, int diagonalstyle_in, int use_shared_arrays_in,
                                          double rmin0_in, int switch_flag_in, int bzero_flag_in,
                                          double *cutoff_array, std::vector<std::string> *species,
                                          std::vector<double> *weights);

    // SOAP and Xi: not provided by this library (throw std::invalid_argument)
    static DescriptorKind *initDescriptor(AvailableDescriptor availableDescriptorKind, int n_max, int l_max,
                                          double cutoff, std::vector<std::string> &species,
                                          std::string radial_basis, double eta);
    static DescriptorKind *initDescriptor(AvailableDescriptor availableDescriptorKind, int q, double cutoff,
                                          std::vector<std::string> &species, std::string &radial_basis);
};

#endif  // LIBDESCRIPTOR_B200_CXX_DESCRIPTORS_HPP_
