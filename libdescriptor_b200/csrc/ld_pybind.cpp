// ld_pybind.cpp -- Python module `_libdescriptor`: the reference's Python
// surface (python_bindings/python_bindings.cpp:50-556) over the C ABI of
// libldb200.so, plus device-pointer entry points for the torch wrapper.
//
// Same names, argument order, dtypes (int32 / float64, C-contiguous,
// force-cast) and return shapes as the reference module `libdescriptor`.
// Errors raise ValueError (bad arguments / kinds, as the reference's
// std::invalid_argument) or RuntimeError (everything else).
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <cmath>
#include <cstdint>
#include <limits>
#include <memory>
#include <string>
#include <vector>

#include "ld_fd.h"
#include "libdescriptor_b200.h"

extern "C" int ld_bs_info(const ld_descriptor *d, long long *inner_fwd, long long *inner_vjp, int *tasks_fwd,
                          int *tasks_vjp, int *nU, int *nL, int *ntrip, int *nZ);

namespace py = pybind11;

using IArr = py::array_t<int, py::array::c_style | py::array::forcecast>;
using DArr = py::array_t<double, py::array::c_style | py::array::forcecast>;

namespace {

void check(int rc) {
    if (rc == LD_OK) return;
    const std::string msg = ld_error_message();
    if (rc == LD_ERR_INVALID_ARG || rc == LD_ERR_INVALID_KIND) throw py::value_error(msg);
    throw std::runtime_error(msg);
}

// A float64 result array.  From 64 KiB up to 64 MiB it lives in the
// library's pinned host blocks (returned to them when the array is freed):
// the device writes there at the link's rate, where the copy into a fresh
// pageable array is bound by its page faults.  Otherwise, or when no pinned
// memory can be had, an ordinary numpy array.
py::array_t<double> result_array(std::vector<py::ssize_t> shape) {
    size_t n = 1;
    for (auto e : shape) n *= (size_t)std::max<py::ssize_t>(e, 0);
    const size_t bytes = n * sizeof(double);
    if (bytes >= (64u << 10) && bytes <= (64u << 20)) {
        void *p = nullptr;
        if (ld_host_alloc(bytes, &p) == LD_OK && p) {
            py::capsule owner(p, [](void *q) { ld_host_free(q); });
            return py::array_t<double>(shape, static_cast<double *>(p), owner);
        }
    }
    return py::array_t<double>(shape);
}

std::vector<py::ssize_t> coords_shape(const DArr &coords) {
    return {coords.shape(0), coords.ndim() > 1 ? coords.shape(1) : (py::ssize_t)1};
}

struct Kind {
    int kind = 0;  // AvailableDescriptor
    std::string param_file;
    std::shared_ptr<ld_descriptor> h;
    int width() const {
        if (!h) return -1;
        int w = 0;
        ld_width(h.get(), &w);
        return w;
    }
    ld_descriptor *get() const {
        if (!h) throw py::value_error("descriptor is empty: initialise it with init_descriptor(kind, ...)");
        return h.get();
    }
};

Kind adopt(ld_descriptor *d, int kind) {
    Kind k;
    k.kind = kind;
    k.h = std::shared_ptr<ld_descriptor>(d, [](ld_descriptor *p) { ld_destroy(p); });
    return k;
}

std::vector<int> sf_codes(const std::vector<std::string> &types) {
    std::vector<int> c;
    for (auto &t : types) {
        if (t == "g1") c.push_back(1);
        else if (t == "g2") c.push_back(2);
        else if (t == "g3") c.push_back(3);
        else if (t == "g4") c.push_back(4);
        else if (t == "g5") c.push_back(5);
        else throw py::value_error("unknown symmetry function type '" + t + "' (expected g1..g5)");
    }
    return c;
}

// The reference binds the cutoff as `double *`: a Python float (or the first
// element of a sequence / array) is the value replicated for every pair.
double first_cutoff(const py::object &c) {
    if (py::isinstance<py::float_>(c) || py::isinstance<py::int_>(c)) return c.cast<double>();
    DArr a = DArr::ensure(c);
    if (!a || a.size() == 0) throw py::value_error("cutoff must be a float or a non-empty sequence");
    return a.data()[0];
}

struct NeighListPy {
    std::vector<int> counts, flat;
    std::vector<long long> begin;
    double cutoff = 0.0;
    int n = 0;
};

}  // namespace

PYBIND11_MODULE(_libdescriptor, m) {
    m.doc() = "B200-native libdescriptor hot path (symmetry functions, bispectrum, VJP)";

    py::class_<Kind>(m, "DescriptorKind")
        .def(py::init<>())
        .def_static("init_descriptor", [](int kind) {
            if (kind < 0 || kind > 3) throw py::value_error("Descriptor kind not implemented yet");
            Kind k;
            k.kind = kind;
            return k;
        })
        .def_static("init_descriptor", [](std::string &file, int kind) {
            ld_descriptor *d = nullptr;
            check(ld_create_from_file(&d, file.c_str(), kind));
            Kind k = adopt(d, kind);
            k.param_file = file;
            return k;
        })
        .def_static("init_descriptor",
                    [](int kind, std::vector<std::string> species, std::string cutoff_function,
                       py::object cutoff, std::vector<std::string> types, std::vector<int> sizes,
                       std::vector<double> params) {
                        if (kind != LD_KIND_SYMMETRY_FUNCTIONS)
                            throw py::value_error("these parameters initialise symmetry functions only");
                        (void)cutoff_function;
                        const int ns = (int)species.size();
                        // the direct init replicates cutoff[0] for every pair
                        // (src/Descriptors.cpp:585)
                        std::vector<double> cm((size_t)ns * ns, first_cutoff(cutoff));
                        auto codes = sf_codes(types);
                        if (sizes.size() != 2 * codes.size()) throw py::value_error("sizes must hold (rows, cols) per type");
                        ld_descriptor *d = nullptr;
                        check(ld_create_symmetry_functions(&d, ns, cm.data(), (int)codes.size(), codes.data(),
                                                           sizes.data(), params.data()));
                        return adopt(d, kind);
                    })
        .def_static("init_descriptor",
                    [](int kind, double rfac0, int twojmax, int diagonalstyle, int use_shared_arrays, double rmin0,
                       int switch_flag, int bzero_flag, py::object cutoff, std::vector<std::string> species,
                       std::vector<double> weights) {
                        if (kind != LD_KIND_BISPECTRUM)
                            throw py::value_error("these parameters initialise the bispectrum only");
                        const int ns = (int)species.size();
                        if ((int)weights.size() < ns) throw py::value_error("one weight per species is required");
                        std::vector<double> cm((size_t)ns * ns, first_cutoff(cutoff));
                        ld_descriptor *d = nullptr;
                        check(ld_create_bispectrum(&d, rfac0, twojmax, diagonalstyle, use_shared_arrays, rmin0,
                                                   switch_flag, bzero_flag, ns, cm.data(), weights.data()));
                        return adopt(d, kind);
                    })
        .def_static("init_descriptor",
                    [](int kind, int, double, std::vector<std::string> &, std::string &) -> Kind {
                        throw py::value_error("Xi descriptor is not part of this library (out of scope)");
                    })
        .def_static("init_descriptor",
                    [](int kind, int, int, double, std::vector<std::string> &, std::string, double) -> Kind {
                        throw py::value_error("SOAP descriptor is not part of this library (out of scope)");
                    })
        .def("compute",
             [](Kind &ds, int index, IArr species, IArr neighbors, DArr coords) {
                 const int w = ds.width();
                 py::array_t<double> out(w);
                 check(ld_compute_single_atom(ds.get(), index, (int)(coords.size() / 3), species.data(),
                                              neighbors.data(), (int)neighbors.size(), coords.data(),
                                              out.mutable_data()));
                 return out;
             })
        .def_readwrite("param_file", &Kind::param_file)
        .def_readwrite("kind", &Kind::kind)
        .def_property_readonly("width", &Kind::width)
        .def("__repr__", [](const Kind &k) {
            return "<DescriptorKind kind=" + std::to_string(k.kind) + " width=" + std::to_string(k.width()) + ">";
        });

    m.def("compute_single_atom", [](Kind &ds, int index, IArr species, IArr neighbors, DArr coords) {
        py::array_t<double> out(ds.width());
        check(ld_compute_single_atom(ds.get(), index, (int)(coords.size() / 3), species.data(), neighbors.data(),
                                     (int)neighbors.size(), coords.data(), out.mutable_data()));
        return out;
    });

    m.def("compute", [](Kind &ds, int n_atoms, IArr species, IArr neighbors, IArr number_of_neighbors, DArr coords) {
        if ((int)number_of_neighbors.size() < n_atoms) throw py::value_error("number_of_neighbors shorter than n_atoms");
        auto out = result_array({n_atoms, ds.width()});
        check(ld_compute(ds.get(), n_atoms, (int)(coords.size() / 3), species.data(), neighbors.data(),
                         number_of_neighbors.data(), coords.data(), out.mutable_data()));
        return out;
    });

    m.def("compute_batch", [](Kind &ds, IArr n_atoms, IArr config_ptr, IArr species, IArr neighbors,
                              IArr number_of_neighbors, DArr coords) {
        const int nc = (int)n_atoms.size();
        long long tot = 0;
        for (int c = 0; c < nc; ++c) tot += n_atoms.data()[c];
        auto out = result_array({(py::ssize_t)tot, (py::ssize_t)ds.width()});
        check(ld_compute_batch(ds.get(), nc, n_atoms.data(), config_ptr.data(), (int)(coords.size() / 3),
                               species.data(), neighbors.data(), number_of_neighbors.data(), coords.data(),
                               out.mutable_data()));
        return out;
    });

    m.def("gradient_single_atom",
          [](Kind &ds, int index, IArr species, IArr neighbors, DArr coords, DArr desc, DArr dE_ddesc) {
              (void)desc;
              py::array_t<double> out({coords.shape(0), coords.ndim() > 1 ? coords.shape(1) : (py::ssize_t)1});
              check(ld_gradient_single_atom(ds.get(), index, (int)(coords.size() / 3), species.data(),
                                            neighbors.data(), (int)neighbors.size(), coords.data(),
                                            dE_ddesc.data(), out.mutable_data(), nullptr));
              return out;
          });

    m.def("gradient", [](Kind &ds, int n_atoms, IArr species, IArr neighbors, IArr number_of_neighbors, DArr coords,
                         DArr desc, DArr dE_ddesc) {
        (void)desc;  // recomputed on the device in the same pass
        if ((long long)dE_ddesc.size() < (long long)n_atoms * ds.width())
            throw py::value_error("dE_ddesc must hold n_atoms * width values");
        auto out = result_array(coords_shape(coords));
        check(ld_gradient(ds.get(), n_atoms, (int)(coords.size() / 3), species.data(), neighbors.data(),
                          number_of_neighbors.data(), coords.data(), dE_ddesc.data(), out.mutable_data(), nullptr));
        return out;
    });

    // dL/d(parameters) of a symmetry-function descriptor, in the flat layout
    // of the parameters given at init
    m.def("gradient_params", [](Kind &ds, int n_atoms, IArr species, IArr neighbors, IArr number_of_neighbors,
                                DArr coords, DArr dE_ddesc) {
        if ((long long)dE_ddesc.size() < (long long)n_atoms * ds.width())
            throw py::value_error("dE_ddesc must hold n_atoms * width values");
        int np = 0;
        check(ld_num_params(ds.get(), &np));
        py::array_t<double> out(std::max(np, 0));
        check(ld_gradient_params(ds.get(), n_atoms, (int)(coords.size() / 3), species.data(), neighbors.data(),
                                 number_of_neighbors.data(), coords.data(), dE_ddesc.data(), out.mutable_data(), np));
        return out;
    });

    // desc + VJP in one fused pass (host buffers): returns (desc, gradient)
    m.def("compute_and_gradient", [](Kind &ds, int n_atoms, IArr species, IArr neighbors, IArr number_of_neighbors,
                                     DArr coords, DArr dE_ddesc) {
        if ((long long)dE_ddesc.size() < (long long)n_atoms * ds.width())
            throw py::value_error("dE_ddesc must hold n_atoms * width values");
        auto desc = result_array({n_atoms, ds.width()});
        auto out = result_array(coords_shape(coords));
        {
            py::gil_scoped_release nogil;
            check(ld_gradient(ds.get(), n_atoms, (int)(coords.size() / 3), species.data(), neighbors.data(),
                              number_of_neighbors.data(), coords.data(), dE_ddesc.data(), out.mutable_data(),
                              desc.mutable_data()));
        }
        return py::make_tuple(desc, out);
    });

    m.def("gradient_batch", [](Kind &ds, IArr n_atoms, IArr config_ptr, IArr species, IArr neighbors,
                               IArr number_of_neighbors, DArr coords, DArr desc, DArr dE_ddesc) {
        (void)desc;
        auto out = result_array(coords_shape(coords));
        check(ld_gradient_batch(ds.get(), (int)n_atoms.size(), n_atoms.data(), config_ptr.data(),
                                (int)(coords.size() / 3), species.data(), neighbors.data(),
                                number_of_neighbors.data(), coords.data(), dE_ddesc.data(), out.mutable_data(),
                                nullptr));
        return out;
    });

    m.def("jacobian", [](Kind &ds, int n_atoms, IArr species, IArr neighbors, IArr number_of_neighbors, DArr coords) {
        const py::ssize_t rows = (py::ssize_t)ds.width() * n_atoms;
        py::array_t<double> out({rows, (py::ssize_t)coords.size()});
        check(ld_jacobian(ds.get(), n_atoms, (int)(coords.size() / 3), species.data(), neighbors.data(),
                          number_of_neighbors.data(), coords.data(), out.mutable_data()));
        return out;
    });

    m.def("num_gradient_single_atom", [](Kind &ds, int index, IArr species, IArr neighbors, DArr coords,
                                         DArr dE_ddesc) {
        const int n_total = (int)(coords.size() / 3);
        const int w = ds.width();
        std::vector<double> x(coords.data(), coords.data() + coords.size());
        auto f = [&](double *xx, double *yy) {
            check(ld_compute_single_atom(ds.get(), index, n_total, species.data(), neighbors.data(),
                                         (int)neighbors.size(), xx, yy));
        };
        py::array_t<double> out(3);
        std::vector<double> dd;
        for (int d = 0; d < 3; ++d) {
            ldb::fd8(f, x, index * 3 + d, w, dd);
            double s = 0.0;
            for (int c = 0; c < w; ++c) s += dE_ddesc.data()[c] * dd[c];
            out.mutable_data()[d] = s;
        }
        return out;
    });

    // ---- neighbour lists (KLIFF-derived builder of the reference)
    py::class_<NeighListPy>(m, "NeighList")
        .def(py::init<>())
        .def("build",
             [](NeighListPy &self, DArr coords, double influence_distance, DArr cutoffs, IArr need_neigh) {
                 const int n = (int)std::min<py::ssize_t>(coords.size() / 3, need_neigh.size());
                 double cut = cutoffs.size() ? cutoffs.data()[0] : influence_distance;
                 self.counts.assign(n, 0);
                 long long nnz = 0;
                 int rc = ld_build_neighbor_list(coords.data(), n, cut, need_neigh.data(), n, self.counts.data(),
                                                 nullptr, &nnz);
                 if (rc) throw std::runtime_error("Cell size too large! (partilces fly away) or\nCollision of atoms happened!");
                 self.flat.assign(nnz, 0);
                 check(ld_build_neighbor_list(coords.data(), n, cut, need_neigh.data(), n, self.counts.data(),
                                              self.flat.data(), &nnz));
                 self.begin.assign(n + 1, 0);
                 for (int a = 0; a < n; ++a) self.begin[a + 1] = self.begin[a] + self.counts[a];
                 self.cutoff = cut;
                 self.n = n;
             },
             py::arg("coords"), py::arg("influence_distance"), py::arg("cutoffs"), py::arg("need_neigh"))
        .def("get_neigh",
             [](NeighListPy &self, DArr cutoffs, int neighbor_list_index, int particle_number) {
                 if (neighbor_list_index != 0)
                     throw std::runtime_error("neighbor_list_index = " + std::to_string(neighbor_list_index) +
                                              " >= self.numberOfNeighborLists = 1");
                 if (cutoffs.size() && cutoffs.data()[0] > self.cutoff + 1e-10)
                     throw std::runtime_error("cutoffs_data[neighbor_list_index] > self.lists[neighbor_list_index].cutoff");
                 if (particle_number < 0 || particle_number >= self.n)
                     throw std::runtime_error("particle_number = " + std::to_string(particle_number) + " < 0!");
                 const int c = self.counts[particle_number];
                 py::array_t<int> arr(c);
                 for (int k = 0; k < c; ++k) arr.mutable_data()[k] = self.flat[self.begin[particle_number] + k];
                 return py::make_tuple(c, arr);
             },
             py::arg("cutoffs"), py::arg("neighbor_list_index"), py::arg("particle_number"));

    m.def("create", []() { return NeighListPy(); });

    m.def("create_paddings",
          [](double influence_distance, DArr cell, IArr pbc, DArr coords, IArr species) {
              const int n = (int)std::min<py::ssize_t>(coords.size() / 3, species.size());
              int np = 0;
              check(ld_create_paddings(influence_distance, cell.data(), pbc.data(), coords.data(), species.data(), n,
                                       &np, nullptr, nullptr, nullptr));
              py::array_t<double> pc({(py::ssize_t)np, (py::ssize_t)3});
              py::array_t<int> ps(np), pi(np);
              check(ld_create_paddings(influence_distance, cell.data(), pbc.data(), coords.data(), species.data(),
                                       n, &np, pc.mutable_data(), ps.mutable_data(), pi.mutable_data()));
              return py::make_tuple(pc, ps, pi);
          },
          py::arg("influence_distance"), py::arg("cell"), py::arg("pbc"), py::arg("coords"), py::arg("species"));

    // ---- device-pointer entry points (torch wrapper, batching, serving)
    m.def("_compute_dev", [](Kind &ds, int n_rows, std::uintptr_t row_centre, std::uintptr_t species,
                             std::uintptr_t nbl, std::uintptr_t off, int max_neigh, std::uintptr_t coords,
                             std::uintptr_t desc, std::uintptr_t stream) {
        check(ld_compute_dev(ds.get(), n_rows, (const int *)row_centre, (const int *)species, (const int *)nbl,
                             (const long long *)off, max_neigh, (const double *)coords, (double *)desc,
                             (ld_stream)stream));
    });
    m.def("_gradient_dev", [](Kind &ds, int n_rows, std::uintptr_t row_centre, std::uintptr_t species,
                              std::uintptr_t nbl, std::uintptr_t off, int max_neigh, std::uintptr_t coords,
                              std::uintptr_t dE, std::uintptr_t dcoords, std::uintptr_t desc, std::uintptr_t image,
                              std::uintptr_t stream) {
        check(ld_gradient_dev(ds.get(), n_rows, (const int *)row_centre, (const int *)species, (const int *)nbl,
                              (const long long *)off, max_neigh, (const double *)coords, (const double *)dE,
                              (double *)dcoords, (double *)desc, (const int *)image, (ld_stream)stream));
    });
    m.def("_compute_rows_dev", [](Kind &ds, int n_rows, std::uintptr_t row_centre, std::uintptr_t nbl_begin,
                                  std::uintptr_t species, std::uintptr_t nbl, std::uintptr_t off, int max_neigh,
                                  std::uintptr_t coords, std::uintptr_t desc, std::uintptr_t work,
                                  std::size_t work_bytes, std::uintptr_t stream) {
        check(ld_compute_rows_dev(ds.get(), n_rows, (const int *)row_centre, (const long long *)nbl_begin,
                                  (const int *)species, (const int *)nbl, (const long long *)off, max_neigh,
                                  (const double *)coords, (double *)desc, (void *)work, work_bytes,
                                  (ld_stream)stream));
    });
    m.def("_gradient_rows_dev", [](Kind &ds, int n_rows, std::uintptr_t row_centre, std::uintptr_t nbl_begin,
                                   std::uintptr_t species, std::uintptr_t nbl, std::uintptr_t off, int max_neigh,
                                   std::uintptr_t coords, std::uintptr_t dE, std::uintptr_t dcoords,
                                   std::uintptr_t desc, std::uintptr_t image, std::uintptr_t work,
                                   std::size_t work_bytes, std::uintptr_t stream) {
        check(ld_gradient_rows_dev(ds.get(), n_rows, (const int *)row_centre, (const long long *)nbl_begin,
                                   (const int *)species, (const int *)nbl, (const long long *)off, max_neigh,
                                   (const double *)coords, (const double *)dE, (double *)dcoords, (double *)desc,
                                   (const int *)image, (void *)work, work_bytes, (ld_stream)stream));
    });
    m.def("_rows_work_bytes", [](Kind &ds, int n_rows, bool vjp) {
        std::size_t b = 0;
        check(ld_rows_work_bytes(ds.get(), n_rows, vjp ? 1 : 0, &b));
        return b;
    });
    m.def("_stage_bytes", [](int n, int nt, long long nnz, int width) {
        std::size_t b = 0;
        check(ld_stage_bytes(n, nt, nnz, width, &b));
        return b;
    });
    m.def("_stage_request", [](int n, int nt, long long nnz, int width, int row0, int atom0, long long entry0,
                               DArr coords, IArr species, IArr image, IArr nbl, IArr counts, DArr dE,
                               std::uintptr_t staging, std::size_t staging_bytes, std::uintptr_t d_coords,
                               std::uintptr_t d_species, std::uintptr_t d_image, std::uintptr_t d_nbl,
                               std::uintptr_t d_centre, std::uintptr_t d_begin, std::uintptr_t d_counts,
                               std::uintptr_t d_dE, std::uintptr_t stream) {
        if ((long long)coords.size() < 3LL * nt || (long long)species.size() < nt || (long long)image.size() < nt ||
            (long long)nbl.size() < nnz || (long long)counts.size() < n || (long long)dE.size() < (long long)n * width)
            throw py::value_error("_stage_request: arrays shorter than the stated sizes");
        int rc;
        {
            py::gil_scoped_release nogil;
            rc = ld_stage_request(n, nt, nnz, width, row0, atom0, entry0, coords.data(), species.data(),
                                  image.data(), nnz ? nbl.data() : nullptr, counts.data(), dE.data(),
                                  (void *)staging, staging_bytes, (double *)d_coords, (int *)d_species,
                                  (int *)d_image, (int *)d_nbl, (int *)d_centre, (long long *)d_begin,
                                  (int *)d_counts, (double *)d_dE, (ld_stream)stream);
        }
        check(rc);
    });
    m.def("_stage_pack", [](int n, int nt, long long nnz, int width, int row0, int atom0, long long entry0,
                            DArr coords, IArr species, IArr image, IArr nbl, IArr counts, DArr dE,
                            std::uintptr_t staging, std::size_t staging_bytes) {
        if ((long long)coords.size() < 3LL * nt || (long long)species.size() < nt || (long long)image.size() < nt ||
            (long long)nbl.size() < nnz || (long long)counts.size() < n || (long long)dE.size() < (long long)n * width)
            throw py::value_error("_stage_pack: arrays shorter than the stated sizes");
        int rc;
        {
            py::gil_scoped_release nogil;
            rc = ld_stage_pack(n, nt, nnz, width, row0, atom0, entry0, coords.data(), species.data(), image.data(),
                               nnz ? nbl.data() : nullptr, counts.data(), dE.data(), (void *)staging, staging_bytes);
        }
        check(rc);
    });
    m.def("_stage_pack_fields", [](int n, int nt, long long nnz, int width, int row0, int atom0, long long entry0,
                                   DArr coords, IArr species, IArr image, IArr nbl, IArr counts, DArr dE,
                                   std::vector<std::uintptr_t> out) {
        if ((long long)coords.size() < 3LL * nt || (long long)species.size() < nt || (long long)image.size() < nt ||
            (long long)nbl.size() < nnz || (long long)counts.size() < n || (long long)dE.size() < (long long)n * width)
            throw py::value_error("_stage_pack_fields: arrays shorter than the stated sizes");
        if (out.size() != 8) throw py::value_error("_stage_pack_fields: 8 output fields");
        int rc;
        {
            py::gil_scoped_release nogil;
            rc = ld_stage_pack_fields(n, nt, nnz, width, row0, atom0, entry0, coords.data(), species.data(),
                                      image.data(), nnz ? nbl.data() : nullptr, counts.data(), dE.data(),
                                      (double *)out[0], (int *)out[1], (int *)out[2], (int *)out[3], (int *)out[4],
                                      (long long *)out[5], (int *)out[6], (double *)out[7]);
        }
        check(rc);
    });
    m.def("_stage_upload_fields", [](std::vector<std::uintptr_t> src, std::vector<std::uintptr_t> dst,
                                     std::vector<std::size_t> bytes, std::uintptr_t stream) {
        if (src.size() != dst.size() || src.size() != bytes.size())
            throw py::value_error("_stage_upload_fields: src, dst and bytes differ in length");
        std::vector<const void *> s(src.size());
        std::vector<void *> d(dst.size());
        for (size_t i = 0; i < src.size(); ++i) {
            s[i] = (const void *)src[i];
            d[i] = (void *)dst[i];
        }
        check(ld_stage_upload_fields((int)src.size(), s.data(), d.data(), bytes.data(), (ld_stream)stream));
    });
    m.def("_stage_upload", [](int n, int nt, long long nnz, int width, int row0, int atom0, long long entry0,
                              std::uintptr_t staging, std::size_t staging_bytes, std::uintptr_t d_coords,
                              std::uintptr_t d_species, std::uintptr_t d_image, std::uintptr_t d_nbl,
                              std::uintptr_t d_centre, std::uintptr_t d_begin, std::uintptr_t d_counts,
                              std::uintptr_t d_dE, std::uintptr_t stream) {
        check(ld_stage_upload(n, nt, nnz, width, row0, atom0, entry0, (void *)staging, staging_bytes,
                              (double *)d_coords, (int *)d_species, (int *)d_image, (int *)d_nbl, (int *)d_centre,
                              (long long *)d_begin, (int *)d_counts, (double *)d_dE, (ld_stream)stream));
    });
    m.def("_create_paddings_dev", [](double cutoff, DArr cell, IArr pbc, std::uintptr_t coords, std::uintptr_t species,
                                     int n_atoms, int max_pad, std::uintptr_t pc, std::uintptr_t ps, std::uintptr_t pi,
                                     std::uintptr_t stream) {
        if (cell.size() != 9 || pbc.size() != 3) throw py::value_error("cell must have 9 values and pbc 3");
        int n = 0, rc;
        {
            py::gil_scoped_release nogil;
            rc = ld_create_paddings_dev(cutoff, cell.data(), pbc.data(), (const double *)coords, (const int *)species,
                                        n_atoms, max_pad, (double *)pc, (int *)ps, (int *)pi, &n, (ld_stream)stream);
        }
        check(rc);
        return n;
    });
    m.def("_build_neighbor_list_dev", [](std::uintptr_t coords, int n_total, double cutoff, std::uintptr_t need,
                                         int n_query, std::uintptr_t counts, std::uintptr_t off, long long max_nnz,
                                         std::uintptr_t nbl, std::uintptr_t stream) {
        long long nnz = 0;
        int mx = 0, rc;
        {
            py::gil_scoped_release nogil;
            rc = ld_build_neighbor_list_dev((const double *)coords, n_total, cutoff, (const int *)need, n_query,
                                            (int *)counts, (long long *)off, max_nnz, (int *)nbl, &nnz, &mx,
                                            (ld_stream)stream);
        }
        check(rc);
        return py::make_tuple(nnz, mx);
    });
    m.def("_set_tuning", [](Kind &ds, int key, int value) { check(ld_set_tuning(ds.get(), key, value)); });
    m.def("_get_tuning", [](Kind &ds, int key) {
        int v = 0;
        check(ld_get_tuning(ds.get(), key, &v));
        return v;
    });
    m.def("_neighbor_offsets_dev", [](Kind &ds, int n_rows, std::uintptr_t counts, std::uintptr_t off,
                                      bool want_max, std::uintptr_t stream) {
        int mx = 0;
        check(ld_neighbor_offsets_dev(ds.get(), n_rows, (const int *)counts, (long long *)off,
                                      want_max ? &mx : nullptr, (ld_stream)stream));
        return mx;
    });
    m.def("_sync_status", [](Kind &ds, std::uintptr_t stream) { check(ld_sync_status(ds.get(), (ld_stream)stream)); });
    m.def("_launch_count", []() { return ld_launch_count(); });
    m.def("_measure_fp64_peak", [](int iters) {
        double t = 0;
        check(ld_measure_fp64_peak(iters, &t));
        return t;
    });
    m.def("_measure_fp64_op_cost", [](int op, int iters, double tflops) {
        double w = 0;
        check(ld_measure_fp64_op_cost(op, iters, tflops, &w));
        return w;
    });
    m.def("_bs_info", [](Kind &ds) {
        long long f = 0, v = 0;
        int tf = 0, tv = 0, nU = 0, nL = 0, nt = 0, nZ = 0;
        check(ld_bs_info(ds.get(), &f, &v, &tf, &tv, &nU, &nL, &nt, &nZ));
        py::dict d;
        d["inner_fwd"] = f;
        d["inner_vjp"] = v;
        d["tasks_fwd"] = tf;
        d["tasks_vjp"] = tv;
        d["nU"] = nU;
        d["nL"] = nL;
        d["ntrip"] = nt;
        d["nZ"] = nZ;
        return d;
    });
}
