// call_site.cpp -- a caller of libdescriptor's C++ driver API, written the
// way a model driver calls the reference (#include "Descriptors.hpp",
// DescriptorKind::initDescriptor, the free functions of namespace
// Descriptor), built against this library's include/cxx/Descriptors.hpp and
// linked with libldb200_cxx.so.  Test input: a case directory written by
// tests/test_cxx_shim.py; every result is written back there as raw float64.
//
//   call_site <case dir>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "Descriptors.hpp"

template <class T>
static std::vector<T> load(const std::string &path, size_t n) {
    std::vector<T> v(n);
    std::ifstream f(path, std::ios::binary);
    if (!f.read(reinterpret_cast<char *>(v.data()), (std::streamsize)(n * sizeof(T))))
        throw std::runtime_error("cannot read " + path);
    return v;
}

static void save(const std::string &path, const std::vector<double> &v) {
    std::ofstream f(path, std::ios::binary);
    f.write(reinterpret_cast<const char *>(v.data()), (std::streamsize)(v.size() * sizeof(double)));
}

int main(int argc, char **argv) {
    if (argc != 2) {
        std::cerr << "usage: call_site <case dir>\n";
        return 2;
    }
    const std::string dir = argv[1];
    std::ifstream meta(dir + "/meta.txt");
    std::string kind_name;
    int n_atoms = 0, n_total = 0, index = 0;
    long long nnz = 0;
    meta >> kind_name >> n_atoms >> n_total >> nnz >> index;
    auto species = load<int>(dir + "/species.i32", n_total);
    auto nbl = load<int>(dir + "/nbl.i32", nnz);
    auto counts = load<int>(dir + "/counts.i32", n_atoms);
    auto coords = load<double>(dir + "/coords.f64", 3 * (size_t)n_total);

    Descriptor::DescriptorKind *kind = nullptr;
    std::vector<std::string> names;
    if (kind_name == "sf") {
        int ns = 0, nt = 0, np = 0;
        double cutoff = 0;
        meta >> ns;
        names.resize(ns);
        for (auto &s : names) meta >> s;
        meta >> cutoff >> nt;
        std::vector<std::string> types(nt);
        for (auto &t : types) meta >> t;
        std::vector<int> sizes(2 * nt);
        for (auto &s : sizes) meta >> s;
        meta >> np;
        std::vector<double> params(np);
        for (auto &p : params) meta >> p;
        std::string cutoff_function = "cos";
        kind = Descriptor::DescriptorKind::initDescriptor(Descriptor::KindSymmetryFunctions, &names,
                                                         &cutoff_function, &cutoff, &types, &sizes, &params);
    } else if (kind_name == "bs") {
        double rfac0, rmin0, cutoff;
        int twojmax, style, switch_flag, bzero_flag, ns;
        meta >> rfac0 >> twojmax >> style >> rmin0 >> switch_flag >> bzero_flag >> cutoff >> ns;
        names.resize(ns);
        for (auto &s : names) meta >> s;
        std::vector<double> weights(ns);
        for (auto &w : weights) meta >> w;
        kind = Descriptor::DescriptorKind::initDescriptor(Descriptor::KindBispectrum, rfac0, twojmax, style, 0,
                                                         rmin0, switch_flag, bzero_flag, &cutoff, &names, &weights);
    } else {
        // a parameter file: "file <kind> <path>"
        int k = 0;
        std::string path;
        meta >> k >> path;
        kind = Descriptor::DescriptorKind::initDescriptor(path, (Descriptor::AvailableDescriptor)k);
    }
    const int W = kind->width;
    auto dE = load<double>(dir + "/dE.f64", (size_t)n_atoms * W);

    // Descriptor::compute, twice into one buffer: symmetry functions add up,
    // the bispectrum is overwritten
    std::vector<double> desc((size_t)n_atoms * W, 0.0);
    Descriptor::compute(n_atoms, species.data(), nbl.data(), counts.data(), coords.data(), desc.data(), kind);
    save(dir + "/desc.f64", desc);
    Descriptor::compute(n_atoms, species.data(), nbl.data(), counts.data(), coords.data(), desc.data(), kind);
    save(dir + "/desc_twice.f64", desc);

    // Descriptor::compute_batch: the atoms as two configurations of one
    // coordinate arena (centre of row (c, j) = j + config_ptr[c])
    std::vector<int> batch_atoms = {n_atoms / 2, n_atoms - n_atoms / 2}, batch_ptr = {0, n_atoms / 2};
    std::vector<double> desc_b((size_t)n_atoms * W, 0.0);
    Descriptor::compute_batch(2, batch_atoms.data(), batch_ptr.data(), species.data(), nbl.data(), counts.data(),
                              coords.data(), desc_b.data(), kind);
    save(dir + "/desc_batch.f64", desc_b);

    // Descriptor::gradient (caller-zeroed buffers)
    std::vector<double> dcoords(3 * (size_t)n_total, 0.0), desc_g((size_t)n_atoms * W, 0.0);
    Descriptor::gradient(n_atoms, species.data(), nbl.data(), counts.data(), coords.data(), dcoords.data(),
                         desc_g.data(), dE.data(), kind);
    save(dir + "/grad.f64", dcoords);
    save(dir + "/desc_grad.f64", desc_g);

    std::vector<double> dcoords_b(3 * (size_t)n_total, 0.0), desc_gb((size_t)n_atoms * W, 0.0);
    Descriptor::gradient_batch(2, batch_atoms.data(), batch_ptr.data(), species.data(), nbl.data(), counts.data(),
                               coords.data(), dcoords_b.data(), desc_gb.data(), dE.data(), kind);
    save(dir + "/grad_batch.f64", dcoords_b);

    // one centre: its own neighbour list, the reference's per-atom calls
    long long off = 0;
    for (int i = 0; i < index; ++i) off += counts[i];
    int *nb = nbl.data() + off;
    std::vector<double> desc_s(W, 0.0);
    Descriptor::compute_single_atom(index, n_atoms, species.data(), nb, counts[index], coords.data(), desc_s.data(),
                                    kind);
    save(dir + "/desc_single.f64", desc_s);
    std::vector<double> dcoords_s(3 * (size_t)n_total, 0.0), desc_sg(W, 0.0);
    Descriptor::gradient_single_atom(index, n_atoms, species.data(), nb, counts[index], coords.data(),
                                     dcoords_s.data(), desc_sg.data(), dE.data() + (size_t)index * W, kind);
    save(dir + "/grad_single.f64", dcoords_s);
    std::vector<double> num(3, 0.0);
    Descriptor::num_gradient_single_atom(index, n_atoms, species.data(), nb, counts[index], coords.data(),
                                         num.data(), dE.data() + (size_t)index * W, kind);
    save(dir + "/num_grad_single.f64", num);

    // Descriptor::jacobian
    std::vector<double> J((size_t)W * n_atoms * 3 * n_total, 0.0);
    Descriptor::jacobian(n_atoms, n_total, species.data(), nbl.data(), counts.data(), coords.data(), J.data(), kind);
    save(dir + "/jacobian.f64", J);

    std::printf("width %d\n", W);
    delete kind;
    return 0;
}
