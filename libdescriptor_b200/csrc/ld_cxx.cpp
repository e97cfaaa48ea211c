// ld_cxx.cpp -- the C++ driver API of libdescriptor (include/cxx/Descriptors.hpp,
// the reference's include/Descriptors.hpp:19-271 and src/Descriptors.cpp)
// over the C ABI of libldb200.so, built as libldb200_cxx.so.
//
// A kind made by an initDescriptor overload owns an ld_descriptor handle;
// every free function of namespace Descriptor forwards to the matching
// ld_* call and applies the reference's buffer rules on the host:
// symmetry-function descriptors are added into desc and bispectrum
// descriptors overwrite it (SymmetryFunctions::compute accumulates,
// Bispectrum::compute assigns); coordinate gradients and Jacobians are added
// into the caller's buffers (the Enzyme shadows accumulate).  The reference
// never passes the number of coordinate rows; it is taken as one past the
// largest centre or neighbour index, which covers every row the results can
// touch.
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/cxx/Descriptors.hpp"
#include "ld_fd.h"
#include "libdescriptor_b200.h"

namespace {

void check(int rc) {
    if (rc == LD_OK) return;
    const std::string msg = ld_error_message();
    if (rc == LD_ERR_INVALID_ARG || rc == LD_ERR_INVALID_KIND || rc == LD_ERR_PARSE) throw std::invalid_argument(msg);
    throw std::runtime_error(msg);
}

// A descriptor kind served by the B200 library.
class LibraryKind final : public Descriptor::DescriptorKind {
   public:
    ld_descriptor *h = nullptr;

    explicit LibraryKind(ld_descriptor *handle, Descriptor::AvailableDescriptor kind) : h(handle) {
        descriptor_kind = kind;
        int w = 0;
        check(ld_width(h, &w));
        width = w;
    }
    ~LibraryKind() override { ld_destroy(h); }

    // descriptor of one centre (the reference's per-atom virtual,
    // include/Descriptors.hpp:227-233), one single-centre launch
    void compute(int index, int, int *species, int *neighbor_lists, int number_of_neighbors, double *coordinates,
                 double *desc) override;
};

// The kind returned by initDescriptor(kind): no parameters yet.
class EmptyKind final : public Descriptor::DescriptorKind {
   public:
    explicit EmptyKind(Descriptor::AvailableDescriptor kind) { descriptor_kind = kind; }
    void compute(int, int, int *, int *, int, double *, double *) override {
        throw std::logic_error("this descriptor kind was created empty (initDescriptor(kind)) and has no parameters");
    }
};

LibraryKind *library_kind(Descriptor::DescriptorKind *k) {
    if (!k) throw std::invalid_argument("descriptor kind is NULL");
    return dynamic_cast<LibraryKind *>(k);
}

LibraryKind *need_library_kind(Descriptor::DescriptorKind *k) {
    LibraryKind *lk = library_kind(k);
    if (!lk) throw std::invalid_argument("gradients need a descriptor kind made by DescriptorKind::initDescriptor");
    return lk;
}

bool accumulates(const Descriptor::DescriptorKind *k) {
    return k->descriptor_kind == Descriptor::KindSymmetryFunctions;
}

// desc += out (symmetry functions) or desc = out (bispectrum)
void deliver(const Descriptor::DescriptorKind *k, double *desc, const std::vector<double> &out) {
    if (!desc) return;
    if (accumulates(k)) {
        for (size_t i = 0; i < out.size(); ++i) desc[i] += out[i];
    } else {
        std::memcpy(desc, out.data(), out.size() * sizeof(double));
    }
}

void add_into(double *dst, const std::vector<double> &src) {
    for (size_t i = 0; i < src.size(); ++i) dst[i] += src[i];
}

long long total_neighbours(int rows, const int *counts) {
    long long s = 0;
    for (int r = 0; r < rows; ++r) s += counts[r];
    return s;
}

// one past the largest index a call can read: centres and neighbours
int rows_needed(int max_centre, const int *nbl, long long nnz) {
    int m = max_centre;
    for (long long q = 0; q < nnz; ++q) m = std::max(m, nbl[q]);
    return m + 1;
}

void LibraryKind::compute(int index, int, int *species, int *neighbor_lists, int number_of_neighbors,
                          double *coordinates, double *desc) {
    const int n_total = rows_needed(index, neighbor_lists, number_of_neighbors);
    std::vector<double> out(width);
    check(ld_compute_single_atom(h, index, n_total, species, neighbor_lists, number_of_neighbors, coordinates,
                                 out.data()));
    deliver(this, desc, out);
}

}  // namespace

using Descriptor::DescriptorKind;

DescriptorKind::~DescriptorKind() = default;

DescriptorKind *DescriptorKind::initDescriptor(AvailableDescriptor kind) {
    if (kind != KindSymmetryFunctions && kind != KindBispectrum)
        throw std::invalid_argument("Descriptor kind not implemented in this library (SOAP and Xi are not provided)");
    return new EmptyKind(kind);
}

DescriptorKind *DescriptorKind::initDescriptor(std::string &file_name, AvailableDescriptor kind) {
    ld_descriptor *h = nullptr;
    check(ld_create_from_file(&h, file_name.c_str(), (int)kind));
    auto *k = new LibraryKind(h, kind);
    k->descriptor_param_file = file_name;
    return k;
}

DescriptorKind *DescriptorKind::initDescriptor(AvailableDescriptor kind, std::vector<std::string> *species,
                                               std::string *cutoff_function, double *cutoff,
                                               std::vector<std::string> *types, std::vector<int> *sizes,
                                               std::vector<double> *params) {
    if (kind != KindSymmetryFunctions) throw std::invalid_argument("this overload makes symmetry functions");
    if (!species || !cutoff || !types || !sizes || !params) throw std::invalid_argument("NULL argument");
    if (cutoff_function && *cutoff_function != "cos")
        throw std::invalid_argument("cutoff function " + *cutoff_function + " is not supported (cos only)");
    const int ns = (int)species->size();
    std::vector<double> cm((size_t)ns * ns, cutoff[0]);
    std::vector<int> codes;
    for (const auto &t : *types) {
        if (t.size() != 2 || (t[0] != 'g' && t[0] != 'G') || t[1] < '1' || t[1] > '5')
            throw std::invalid_argument("unknown symmetry function type " + t);
        codes.push_back(t[1] - '0');
    }
    if (sizes->size() < 2 * codes.size()) throw std::invalid_argument("symmetry_function_sizes too short");
    ld_descriptor *h = nullptr;
    check(ld_create_symmetry_functions(&h, ns, cm.data(), (int)codes.size(), codes.data(), sizes->data(),
                                       params->data()));
    return new LibraryKind(h, kind);
}

DescriptorKind *DescriptorKind::initDescriptor(AvailableDescriptor kind, double rfac0, int twojmax, int diagonalstyle,
                                               int use_shared_arrays, double rmin0, int switch_flag, int bzero_flag,
                                               double *cutoff, std::vector<std::string> *species,
                                               std::vector<double> *weights) {
    if (kind != KindBispectrum) throw std::invalid_argument("this overload makes the bispectrum");
    if (!cutoff || !species || !weights) throw std::invalid_argument("NULL argument");
    const int ns = (int)species->size();
    if ((int)weights->size() < ns) throw std::invalid_argument("one weight per species is needed");
    std::vector<double> cm((size_t)ns * ns, cutoff[0]);
    ld_descriptor *h = nullptr;
    check(ld_create_bispectrum(&h, rfac0, twojmax, diagonalstyle, use_shared_arrays, rmin0, switch_flag, bzero_flag,
                               ns, cm.data(), weights->data()));
    return new LibraryKind(h, kind);
}

DescriptorKind *DescriptorKind::initDescriptor(AvailableDescriptor, int, int, double, std::vector<std::string> &,
                                               std::string, double) {
    throw std::invalid_argument("SOAP is not provided by this library");
}

DescriptorKind *DescriptorKind::initDescriptor(AvailableDescriptor, int, double, std::vector<std::string> &,
                                               std::string &) {
    throw std::invalid_argument("Xi is not provided by this library");
}

namespace Descriptor {

void compute(int n_atoms, int *species, int *neighbor_list, int *number_of_neighs, double *coordinates, double *desc,
             DescriptorKind *descriptor_kind) {
    LibraryKind *lk = library_kind(descriptor_kind);
    if (!lk) {
        // a caller's own kind: its per-centre compute, rows in order
        int *nb = neighbor_list;
        for (int i = 0; i < n_atoms; ++i) {
            descriptor_kind->compute(i, n_atoms, species, nb, number_of_neighs[i], coordinates,
                                     desc + (size_t)i * descriptor_kind->width);
            nb += number_of_neighs[i];
        }
        return;
    }
    if (n_atoms <= 0) return;
    const long long nnz = total_neighbours(n_atoms, number_of_neighs);
    const int n_total = rows_needed(n_atoms - 1, neighbor_list, nnz);
    std::vector<double> out((size_t)n_atoms * lk->width);
    check(ld_compute(lk->h, n_atoms, n_total, species, neighbor_list, number_of_neighs, coordinates, out.data()));
    deliver(lk, desc, out);
}

void compute_batch(int n_configurations, int *n_atoms, int *config_ptr, int *species, int *neighbor_list,
                   int *number_of_neighs, double *coordinates, double *desc, DescriptorKind *descriptor_kind) {
    int rows = 0, max_centre = -1;
    for (int c = 0; c < n_configurations; ++c) {
        rows += n_atoms[c];
        if (n_atoms[c] > 0) max_centre = std::max(max_centre, config_ptr[c] + n_atoms[c] - 1);
    }
    LibraryKind *lk = library_kind(descriptor_kind);
    if (!lk) {
        int *nb = neighbor_list;
        int r = 0;
        for (int c = 0; c < n_configurations; ++c)
            for (int j = 0; j < n_atoms[c]; ++j, ++r) {
                descriptor_kind->compute(j + config_ptr[c], rows, species, nb, number_of_neighs[r], coordinates,
                                         desc + (size_t)r * descriptor_kind->width);
                nb += number_of_neighs[r];
            }
        return;
    }
    if (rows <= 0) return;
    const long long nnz = total_neighbours(rows, number_of_neighs);
    const int n_total = rows_needed(max_centre, neighbor_list, nnz);
    std::vector<double> out((size_t)rows * lk->width);
    check(ld_compute_batch(lk->h, n_configurations, n_atoms, config_ptr, n_total, species, neighbor_list,
                           number_of_neighs, coordinates, out.data()));
    deliver(lk, desc, out);
}

void compute_single_atom(int index, int n_atoms, int *species, int *neighbor_list, int number_of_neighs,
                         double *coordinates, double *desc, DescriptorKind *descriptor_kind) {
    if (!descriptor_kind) throw std::invalid_argument("descriptor kind is NULL");
    descriptor_kind->compute(index, n_atoms, species, neighbor_list, number_of_neighs, coordinates, desc);
}

void gradient(int n_atoms, int *species, int *neighbor_list, int *number_of_neighs, double *coordinates,
              double *d_coordinates, double *desc, double *dE_dzeta, DescriptorKind *descriptor_to_diff) {
    LibraryKind *lk = need_library_kind(descriptor_to_diff);
    if (n_atoms <= 0) return;
    const long long nnz = total_neighbours(n_atoms, number_of_neighs);
    const int n_total = rows_needed(n_atoms - 1, neighbor_list, nnz);
    std::vector<double> dc((size_t)3 * n_total), out((size_t)n_atoms * lk->width);
    check(ld_gradient(lk->h, n_atoms, n_total, species, neighbor_list, number_of_neighs, coordinates, dE_dzeta,
                      dc.data(), out.data()));
    add_into(d_coordinates, dc);
    deliver(lk, desc, out);
}

void gradient_batch(int n_configurations, int *n_atoms, int *config_ptr, int *species, int *neighbor_list,
                    int *number_of_neighs, double *coordinates, double *d_coordinates, double *desc,
                    double *dE_dzeta, DescriptorKind *descriptor_to_diff) {
    LibraryKind *lk = need_library_kind(descriptor_to_diff);
    int rows = 0, max_centre = -1;
    for (int c = 0; c < n_configurations; ++c) {
        rows += n_atoms[c];
        if (n_atoms[c] > 0) max_centre = std::max(max_centre, config_ptr[c] + n_atoms[c] - 1);
    }
    if (rows <= 0) return;
    const long long nnz = total_neighbours(rows, number_of_neighs);
    const int n_total = rows_needed(max_centre, neighbor_list, nnz);
    std::vector<double> dc((size_t)3 * n_total), out((size_t)rows * lk->width);
    check(ld_gradient_batch(lk->h, n_configurations, n_atoms, config_ptr, n_total, species, neighbor_list,
                            number_of_neighs, coordinates, dE_dzeta, dc.data(), out.data()));
    add_into(d_coordinates, dc);
    deliver(lk, desc, out);
}

void gradient_single_atom(int index, int, int *species, int *neighbor_list, int number_of_neighs,
                          double *coordinates, double *d_coordinates, double *desc, double *dE_dzeta,
                          DescriptorKind *descriptor_to_diff) {
    LibraryKind *lk = need_library_kind(descriptor_to_diff);
    const int n_total = rows_needed(index, neighbor_list, number_of_neighs);
    std::vector<double> dc((size_t)3 * n_total), out(lk->width);
    check(ld_gradient_single_atom(lk->h, index, n_total, species, neighbor_list, number_of_neighs, coordinates,
                                  dE_dzeta, dc.data(), out.data()));
    add_into(d_coordinates, dc);
    deliver(lk, desc, out);
}

void num_gradient_single_atom(int index, int, int *species, int *neighbor_list, int number_of_neighs,
                              double *coordinates, double *d_coordinates, double *dE_dzeta,
                              DescriptorKind *descriptor_to_diff) {
    LibraryKind *lk = need_library_kind(descriptor_to_diff);
    const int n_total = rows_needed(index, neighbor_list, number_of_neighs);
    std::vector<double> x(coordinates, coordinates + (size_t)3 * n_total), dd;
    auto f = [&](double *xx, double *yy) {
        check(ld_compute_single_atom(lk->h, index, n_total, species, neighbor_list, number_of_neighs, xx, yy));
    };
    for (int d = 0; d < 3; ++d) {
        ldb::fd8(f, x, index * 3 + d, lk->width, dd);
        for (int c = 0; c < lk->width; ++c) d_coordinates[d] += dE_dzeta[c] * dd[c];
    }
}

void jacobian(int n_atoms, int n_total_atoms, int *species, int *neighbor_list, int *number_of_neighs,
              double *coordinates, double *J_coordinates, DescriptorKind *descriptor_to_diff) {
    LibraryKind *lk = need_library_kind(descriptor_to_diff);
    if (n_atoms <= 0) return;
    std::vector<double> J((size_t)lk->width * n_atoms * 3 * n_total_atoms);
    check(ld_jacobian(lk->h, n_atoms, n_total_atoms, species, neighbor_list, number_of_neighs, coordinates,
                      J.data()));
    add_into(J_coordinates, J);
}

}  // namespace Descriptor
