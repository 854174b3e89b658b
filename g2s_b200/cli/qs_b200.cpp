// qs_b200: the G2S `qs` command line on the B200 batched engine.
//
// Reads its grids from the G2S data directory (/tmp/G2S/data, or
// $G2S_DATA_DIR) by name like G2S' DataImage::createFromFile, runs the whole
// vector (or -fs) simulation on one GPU through the C ABI and writes the
// simulation and the index image back under the job id, as the reference
// `qs` does (src/qs.cpp:364-2300): <id>.bgrid and id_<id>.bgrid.  The
// arguments follow G2S' own reader (include/utils.hpp:115-138: a flag
// followed by its values) and the flags of src/qs.cpp:356-357,552-760.
//
//   qs_b200 -ti TI [TI2 ...] -di DI -k 1.5 -n 80 -s 100 [-ki K1 [K2 ...]] [-kii KII] [-ii II]
//           [-ni NI] [-kvi KVI] [-fs] [-nV] [-id JOB] [-r REPORT] [-W_CUDA 0]
//
// Flags of the reference that this path does not implement (several
// training images, -ii, -sp, -csim, -cti, -maxNK, ...) end the run with a
// message and status 1; nothing falls back to a CPU path.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <set>
#include <string>
#include <vector>

#include "g2s_b200.h"

namespace {

std::multimap<std::string, std::string> read_args(int argc, char **argv) {
    std::multimap<std::string, std::string> arg;
    int i = 1;
    while (i < argc) {
        if (argv[i][0] == '-') {
            const std::string name = argv[i++];
            bool one = false;
            while (i < argc && argv[i][0] != '-') {
                arg.emplace(name, argv[i++]);
                one = true;
            }
            if (!one) arg.emplace(name, std::string());
        } else {
            ++i;
        }
    }
    return arg;
}

struct Grid {
    int ndim = 0, nvar = 0, encoding = 0;
    unsigned dims[16] = {0};
    std::vector<int> types;
    std::vector<float> data;
    long long cells() const {
        long long c = 1;
        for (int d = 0; d < ndim; ++d) c *= dims[d];
        return c;
    }
};

std::string data_dir() {
    const char *e = std::getenv("G2S_DATA_DIR");
    return e && *e ? std::string(e) : std::string("/tmp/G2S/data");
}

bool load(const std::string &name, Grid &g, FILE *rep) {
    for (const char *ext : {".bgrid.gz", ".bgrid"}) {
        const std::string path = data_dir() + "/" + name + ext;
        FILE *f = std::fopen(path.c_str(), "rb");
        if (!f) continue;
        std::fclose(f);
        long long count = 0;
        g.types.assign(4096, 0);
        if (qsk_bgrid_read(path.c_str(), &g.ndim, g.dims, &g.nvar, g.types.data(), 4096, &g.encoding, nullptr, 0,
                           &count) != QSK_OK)
            break;
        g.types.resize(size_t(g.nvar));
        g.data.resize(size_t(count));
        if (qsk_bgrid_read(path.c_str(), &g.ndim, g.dims, &g.nvar, nullptr, 0, &g.encoding, g.data.data(), count,
                           &count) != QSK_OK)
            break;
        return true;
    }
    std::fprintf(rep, "error: grid '%s' not found or invalid in %s (%s)\n", name.c_str(), data_dir().c_str(),
                 qsk_last_error());
    return false;
}

}  // namespace

int main(int argc, char **argv) {
    auto arg = read_args(argc, argv);
    FILE *rep = stderr;
    if (arg.count("-r") && !arg.find("-r")->second.empty()) {
        FILE *f = std::fopen(arg.find("-r")->second.c_str(), "a");
        if (f) rep = f;
    }
    auto fail = [&](const char *msg) {
        std::fprintf(rep, "error: %s\n", msg);
        if (rep != stderr) std::fclose(rep);
        return 1;
    };
    if (arg.count("-h") || arg.count("--help")) {
        std::printf("qs_b200 -ti TI [TI2 ...] -di DI -k K -n N [N2 ...] -s SEED [-ki K1 ...] [-kii KII] [-ni NI]\n"
                    "        [-kvi KVI] [-ii II] [-fs] [-nV] [-id JOB] [-r REPORT] [-W_CUDA DEVICE]\n");
        return 0;
    }
    static const std::set<std::string> known = {"-ti", "-di", "-dt", "-k", "-n", "-s", "-ki", "-kii", "-ni", "-kvi",
                                                "-ii", "-fs", "-nV", "-id", "-r", "-j", "-W_CUDA", "-W_GPU"};
    for (auto &kv : arg)
        if (!known.count(kv.first)) {
            std::string m = "flag " + kv.first + " is not implemented on the B200 path";
            return fail(m.c_str());
        }
    if (arg.count("-ti") < 1) return fail("-ti is required");
    if (!arg.count("-di")) return fail("-di is required");
    if (!arg.count("-n") && !arg.count("-ni")) return fail("number of neighbours (-n or -ni) is required");

    // training images in the order given (-ti a b ... ; src/qs.cpp reads them so)
    std::vector<Grid> tis;
    for (auto it = arg.equal_range("-ti").first; it != arg.equal_range("-ti").second; ++it) {
        Grid g;
        if (!load(it->second, g, rep)) return fail("training image grid");
        tis.push_back(std::move(g));
    }
    Grid di;
    if (!load(arg.find("-di")->second, di, rep)) return fail("input grid");
    const Grid &ti = tis[0];
    for (const Grid &t : tis)
        if (t.ndim != di.ndim || t.nvar != di.nvar)
            return fail("training images and grid differ in dimensions or variables");

    std::vector<int> nlist;
    for (auto it = arg.equal_range("-n").first; it != arg.equal_range("-n").second; ++it)
        nlist.push_back(std::atoi(it->second.c_str()));
    float k = arg.count("-k") ? float(std::atof(arg.find("-k")->second.c_str())) : NAN;
    unsigned seed = arg.count("-s") ? unsigned(std::strtoul(arg.find("-s")->second.c_str(), nullptr, 10)) : 0u;
    int device = 0;
    for (const char *w : {"-W_CUDA", "-W_GPU"})
        if (arg.count(w) && !arg.find(w)->second.empty()) device = std::atoi(arg.find(w)->second.c_str());
    const std::string job = arg.count("-id") && !arg.find("-id")->second.empty() ? arg.find("-id")->second : "qs_b200";

    qsk_qs_params p;
    std::memset(&p, 0, sizeof(p));
    p.ndim = ti.ndim;
    p.ti_dims = ti.dims;
    p.nvar = ti.nvar;
    p.types = ti.types.data();
    p.ti = ti.data.data();
    p.di_dims = di.dims;
    p.n = nlist.empty() ? 0 : nlist[0];
    if (nlist.size() > 1) {
        p.n_counts = int(nlist.size());
        p.n_per_variable = nlist.data();
    }
    p.k = k;
    p.seed = seed;
    p.no_verbatim = arg.count("-nV") ? 1 : 0;
    p.full_simulation = arg.count("-fs") ? 1 : 0;
    std::vector<unsigned> xdims;
    std::vector<const float *> xptr;
    for (size_t t = 1; t < tis.size(); ++t) {
        for (int d = 0; d < tis[t].ndim; ++d) xdims.push_back(tis[t].dims[d]);
        xptr.push_back(tis[t].data.data());
    }
    if (!xptr.empty()) {
        p.n_extra_tis = int(xptr.size());
        p.extra_ti_dims = xdims.data();
        p.extra_tis = xptr.data();
    }
    Grid ii;
    if (arg.count("-ii")) {
        if (!load(arg.find("-ii")->second, ii, rep)) return fail("-ii grid");
        if (ii.cells() != di.cells()) return fail("-ii grid size differs from -di");
        p.ti_index_image = ii.data.data();
    }

    // kernels: one weight per cell and variable (a one-variable kernel is
    // shared by all variables, as G2S reads it with i % nbVariable)
    std::vector<Grid> kern;
    std::vector<std::vector<float>> kdata;
    std::vector<unsigned> kdims;
    std::vector<const float *> kptr;
    for (auto it = arg.equal_range("-ki").first; it != arg.equal_range("-ki").second; ++it) {
        Grid g;
        if (!load(it->second, g, rep)) return fail("kernel grid");
        if (g.ndim != ti.ndim) return fail("kernel dimensions differ from the training image");
        std::vector<float> w(size_t(g.cells()) * ti.nvar);
        for (long long c = 0; c < g.cells(); ++c)
            for (int v = 0; v < ti.nvar; ++v) w[size_t(c) * ti.nvar + v] = g.data[size_t(c) * g.nvar + (v % g.nvar)];
        for (int d = 0; d < g.ndim; ++d) kdims.push_back(g.dims[d]);
        kdata.push_back(std::move(w));
        kern.push_back(std::move(g));
    }
    for (auto &w : kdata) kptr.push_back(w.data());
    if (kdata.size() == 1) {
        p.kernel_dims = kdims.data();
        p.kernel = kptr[0];
    } else if (kdata.size() > 1) {
        p.n_kernels = int(kdata.size());
        p.kernels_dims = kdims.data();
        p.kernels = kptr.data();
    }
    Grid kii, ni, kvi;
    if (arg.count("-kii")) {
        if (!load(arg.find("-kii")->second, kii, rep)) return fail("-kii grid");
        if (kii.cells() != di.cells()) return fail("-kii grid size differs from -di");
        p.kernel_index_image = kii.data.data();
    }
    if (arg.count("-ni")) {
        if (!load(arg.find("-ni")->second, ni, rep)) return fail("-ni grid");
        if (ni.cells() != di.cells()) return fail("-ni grid size differs from -di");
        p.n_image_vars = ni.nvar;
        p.n_image = ni.data.data();
    }
    if (arg.count("-kvi")) {
        if (!load(arg.find("-kvi")->second, kvi, rep)) return fail("-kvi grid");
        if (kvi.cells() != di.cells() || kvi.nvar != 1) return fail("-kvi needs one value per grid cell");
        p.k_image = kvi.data.data();
    }
    if (std::isnan(p.k) && !p.k_image) return fail("number of candidates (-k) is required");

    std::vector<float> out = di.data;
    const size_t nid = size_t(di.cells()) * (p.full_simulation ? di.nvar : 1);
    std::vector<unsigned> id(nid, 0u);
    auto t0 = std::chrono::high_resolution_clock::now();
    int rc = qsk_simulate(device, &p, out.data(), id.data());
    auto t1 = std::chrono::high_resolution_clock::now();
    if (rc != QSK_OK) {
        std::string m = std::string("simulation failed: ") + qsk_last_error();
        return fail(m.c_str());
    }
    const long long ms = (long long)std::chrono::duration_cast<std::chrono::milliseconds>(t1 - t0).count();
    // same report line as the reference (src/qs.cpp:2229-2235)
    std::fprintf(rep, "compuattion time: %lld ms\n", ms);
    const std::string sim_path = data_dir() + "/" + job + ".bgrid";
    const std::string id_path = data_dir() + "/id_" + job + ".bgrid";
    if (qsk_bgrid_write(sim_path.c_str(), di.ndim, di.dims, di.nvar, di.types.data(), 0, out.data(), 0) != QSK_OK)
        return fail(qsk_last_error());
    std::vector<int> idtypes(size_t(p.full_simulation ? di.nvar : 1), 0);
    if (qsk_bgrid_write(id_path.c_str(), di.ndim, di.dims, int(idtypes.size()), idtypes.data(), 2, id.data(), 0) !=
        QSK_OK)
        return fail(qsk_last_error());
    if (rep != stderr) std::fclose(rep);
    return 0;
}
