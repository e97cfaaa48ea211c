// ref_driver.cpp -- TEST INFRASTRUCTURE ONLY.
//
// A thin extern "C" driver around the REFERENCE's own C++ (compiled from
// the reference source tree by oracle/Makefile into oracle/_ref/).  It lets
// the tests and the CPU baseline run the reference's forward code and its
// neighbour-list builder on the same inputs as the GPU path.  No reference
// source is copied here; this file only calls the reference classes:
//   SymmetryFunctions(...)  include/SymmetryFunctions.hpp:36-41
//   Bispectrum(...)         include/Bispectrum.hpp:117-123 (+ set_species /
//                           set_cutoff / set_weight as done by the direct
//                           init, src/Descriptors.cpp:592-607)
//   DescriptorKind::compute include/Descriptors.hpp:227-233
//   nbl_create_paddings / nbl_build / nbl_get_neigh
//                           python_bindings/neighbor/neighbor_list.h:26-51
//   numdiff::vec_finite_difference_derivative
//                           include/finite_difference.hpp:59-143
// The whole-configuration loops restate Descriptor::compute /
// compute_batch (src/Descriptors.cpp:121-163), which live in a translation
// unit that needs the Enzyme toolchain and so cannot be built here.
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "Bispectrum.hpp"
#include "Descriptors.hpp"
#include "SymmetryFunctions.hpp"
#include "finite_difference.hpp"
#include "neighbor/neighbor_list.h"

// The only symbol of src/Descriptors.cpp the descriptor classes need.
Descriptor::DescriptorKind::~DescriptorKind() = default;

namespace {
struct RefKind {
    int kind = 0;  // 0 = SF, 1 = BS
    // SF construction arguments
    std::vector<std::string> species;
    std::string cutoff_function = "cos";
    std::vector<double> cutoff_matrix;
    std::vector<std::string> types;
    std::vector<int> sizes;
    std::vector<double> params;
    // BS construction arguments
    double rfac0 = 0, rmin0 = 0;
    int twojmax = 0, style = 3, use_shared = 0, switch_flag = 1, bzero_flag = 0;
    std::vector<double> weights;
    // parameter-file construction (SymmetryFunctions(std::string&),
    // src/SymmetryFunctions.cpp:262-407; Bispectrum(std::string&),
    // src/Bispectrum.cpp:848-1007) when set
    std::string file;
    std::vector<Descriptor::DescriptorKind *> inst;

    Descriptor::DescriptorKind *make() {
        if (!file.empty()) {
            std::string f = file;
            if (kind == 0) {
                auto *sf = new SymmetryFunctions(f);
                sf->descriptor_kind = Descriptor::KindSymmetryFunctions;
                return sf;
            }
            auto *bs = new Bispectrum(f);
            bs->descriptor_kind = Descriptor::KindBispectrum;
            return bs;
        }
        if (kind == 0) {
            auto *sf = new SymmetryFunctions(&species, &cutoff_function, cutoff_matrix.data(),
                                             &types, &sizes, &params);
            sf->descriptor_kind = Descriptor::KindSymmetryFunctions;
            return sf;
        }
        auto *bs = new Bispectrum(rfac0, twojmax, style, use_shared, rmin0, switch_flag,
                                  bzero_flag);
        bs->width = bs->get_width();
        bs->set_species((int)species.size());
        bs->set_cutoff("cos", species.size(), cutoff_matrix.data());
        bs->set_weight((int)species.size(), weights.data());
        bs->descriptor_kind = Descriptor::KindBispectrum;
        return bs;
    }
    Descriptor::DescriptorKind *get(int t) {
        while ((int)inst.size() <= t) inst.push_back(make());
        return inst[t];
    }
    ~RefKind() {
        for (auto *p : inst) {
            if (kind == 0) delete static_cast<SymmetryFunctions *>(p);
            else delete static_cast<Bispectrum *>(p);
        }
    }
};

const char *sf_name(int code) {
    static const char *names[] = {"", "g1", "g2", "g3", "g4", "g5"};
    return (code >= 1 && code <= 5) ? names[code] : "";
}
}  // namespace

extern "C" {

void *ref_sf_new(int n_species, const double *cutoff_matrix, int n_types,
                 const int *type_codes, const int *sizes, const double *params) {
    auto *k = new RefKind;
    k->kind = 0;
    for (int s = 0; s < n_species; ++s) k->species.push_back("S" + std::to_string(s));
    k->cutoff_matrix.assign(cutoff_matrix, cutoff_matrix + n_species * n_species);
    size_t np = 0;
    for (int t = 0; t < n_types; ++t) {
        k->types.push_back(sf_name(type_codes[t]));
        k->sizes.push_back(sizes[2 * t]);
        k->sizes.push_back(sizes[2 * t + 1]);
        np += (size_t)sizes[2 * t] * sizes[2 * t + 1];
    }
    k->params.assign(params, params + np);
    k->get(0);
    return k;
}

// A reference descriptor built from a parameter file (kind 0 = symmetry
// functions, 1 = bispectrum); NULL when the reference's reader throws.
void *ref_from_file(const char *path, int kind) {
    auto *k = new RefKind;
    k->kind = kind;
    k->file = path;
    try {
        k->get(0);
    } catch (const std::exception &) {
        k->inst.clear();
        delete k;
        return nullptr;
    }
    return k;
}

void *ref_bs_new(double rfac0, int twojmax, int style, int use_shared, double rmin0,
                 int switch_flag, int bzero_flag, int n_species,
                 const double *cutoff_matrix, const double *weights) {
    auto *k = new RefKind;
    k->kind = 1;
    for (int s = 0; s < n_species; ++s) k->species.push_back("S" + std::to_string(s));
    k->cutoff_matrix.assign(cutoff_matrix, cutoff_matrix + n_species * n_species);
    k->weights.assign(weights, weights + n_species);
    k->rfac0 = rfac0;
    k->twojmax = twojmax;
    k->style = style;
    k->use_shared = use_shared;
    k->rmin0 = rmin0;
    k->switch_flag = switch_flag;
    k->bzero_flag = bzero_flag;
    k->get(0);
    return k;
}

void ref_free(void *h) { delete static_cast<RefKind *>(h); }

int ref_width(void *h) { return static_cast<RefKind *>(h)->get(0)->width; }

// Descriptor::compute / compute_batch layout; n_configs == 0 means a single
// configuration with centres 0..n_atoms[0]-1.  desc is zeroed first (as the
// reference Python binding does, python_bindings.cpp:146-147).
int ref_compute(void *h, int n_configs, const int *n_atoms, const int *config_ptr,
                const int *species, const int *nbl, const int *counts,
                const double *coords, double *desc, int n_threads) {
    auto *k = static_cast<RefKind *>(h);
    std::vector<int> centre;
    if (n_configs <= 0) {
        for (int i = 0; i < n_atoms[0]; ++i) centre.push_back(i);
    } else {
        for (int c = 0; c < n_configs; ++c)
            for (int j = 0; j < n_atoms[c]; ++j) centre.push_back(j + config_ptr[c]);
    }
    const int nrows = (int)centre.size();
    std::vector<long long> off(nrows + 1, 0);
    for (int r = 0; r < nrows; ++r) off[r + 1] = off[r] + counts[r];
    const int width = k->get(0)->width;
    std::memset(desc, 0, sizeof(double) * (size_t)nrows * width);
    if (n_threads < 1) n_threads = 1;
    if (n_threads > nrows) n_threads = nrows > 0 ? nrows : 1;
    for (int t = 0; t < n_threads; ++t) k->get(t);
    auto work = [&](int t) {
        Descriptor::DescriptorKind *dk = k->inst[t];
        const int r0 = (int)((long long)nrows * t / n_threads);
        const int r1 = (int)((long long)nrows * (t + 1) / n_threads);
        for (int r = r0; r < r1; ++r)
            dk->compute(centre[r], nrows, const_cast<int *>(species),
                        const_cast<int *>(nbl + off[r]), counts[r],
                        const_cast<double *>(coords), desc + (size_t)r * width);
    };
    if (n_threads == 1) {
        work(0);
    } else {
        std::vector<std::thread> th;
        for (int t = 0; t < n_threads; ++t) th.emplace_back(work, t);
        for (auto &x : th) x.join();
    }
    return 0;
}

// Descriptor::num_gradient_single_atom (src/Descriptors.cpp:488-518) on the
// reference classes: d/dr_index of (dE . desc_index), 8th-order stencil.
int ref_num_gradient_single_atom(void *h, int index, int n_atoms_total, const int *species,
                                 const int *nbl, int n_neigh, const double *coords,
                                 const double *dE, double *out3) {
    auto *k = static_cast<RefKind *>(h);
    Descriptor::DescriptorKind *dk = k->get(0);
    std::vector<double> x(coords, coords + 3 * (size_t)n_atoms_total);
    auto f = [&](double *xx, double *yy) {
        dk->compute(index, n_atoms_total, const_cast<int *>(species), const_cast<int *>(nbl),
                    n_neigh, xx, yy);
    };
    std::vector<double> dd(dk->width, 0.0);
    for (int d = 0; d < 3; ++d) {
        std::fill(dd.begin(), dd.end(), 0.0);
        numdiff::vec_finite_difference_derivative(f, x.data(), index * 3 + d,
                                                  n_atoms_total * 3, dk->width, dd.data());
        double s = 0.0;
        for (int c = 0; c < dk->width; ++c) s += dE[c] * dd[c];
        out3[d] = s;
    }
    return 0;
}

// nbl_create_paddings; outputs are malloc'd, release with ref_free_buf.
int ref_create_paddings(double cutoff, const double *cell, const int *pbc,
                        const double *coords, const int *species, int n,
                        int *n_pad, double **pad_coords, int **pad_species,
                        int **pad_image) {
    int np = 0;
    std::vector<double> pc;
    std::vector<int> ps, pi;
    int err = nbl_create_paddings(n, cutoff, cell, pbc, coords, species, np, pc, ps, pi);
    if (err) return err;
    *n_pad = np;
    *pad_coords = (double *)std::malloc(sizeof(double) * (pc.size() + 1));
    *pad_species = (int *)std::malloc(sizeof(int) * (ps.size() + 1));
    *pad_image = (int *)std::malloc(sizeof(int) * (pi.size() + 1));
    std::memcpy(*pad_coords, pc.data(), sizeof(double) * pc.size());
    std::memcpy(*pad_species, ps.data(), sizeof(int) * ps.size());
    std::memcpy(*pad_image, pi.data(), sizeof(int) * pi.size());
    return 0;
}

// nbl_build with one cutoff + the flat (numneigh, neighlist) of the atoms
// with need_neigh != 0, as NeighborList.get_numneigh_and_neighlist_1D does
// for contributing atoms (python_package/libdescriptor/neighbor.py:108-154).
int ref_nbl_build(const double *coords, int n, double cutoff, const int *need_neigh,
                  int n_query, int **counts, int **nbl, long long *nnz) {
    NeighList *nl = nullptr;
    nbl_initialize(&nl);
    double cut = cutoff;
    int err = nbl_build(nl, n, coords, cutoff, 1, &cut, need_neigh);
    if (err) {
        nbl_clean(&nl);
        return err;
    }
    std::vector<int> cnt, flat;
    for (int i = 0; i < n_query; ++i) {
        int nn = 0;
        const int *ng = nullptr;
        nbl_get_neigh(nl, 1, &cut, 0, i, &nn, &ng);
        cnt.push_back(nn);
        flat.insert(flat.end(), ng, ng + nn);
    }
    nbl_clean(&nl);
    *counts = (int *)std::malloc(sizeof(int) * (cnt.size() + 1));
    *nbl = (int *)std::malloc(sizeof(int) * (flat.size() + 1));
    std::memcpy(*counts, cnt.data(), sizeof(int) * cnt.size());
    std::memcpy(*nbl, flat.data(), sizeof(int) * flat.size());
    *nnz = (long long)flat.size();
    return 0;
}

void ref_free_buf(void *p) { std::free(p); }

}  // extern "C"
