// auto_qs_b200: the G2S `auto_qs` calibration command line on the B200
// batched engine.
//
// Reads its grids from the G2S data directory (/tmp/G2S/data, or
// $G2S_DATA_DIR) by name, runs the calibration on one GPU through
// qsk_calibrate and writes the three images the reference `auto_qs` writes
// (src/auto_qs.cpp:645-760): im_1_<id> (mean error^(1/p)), im_2_<id>
// (deviation^(0.5/p)), im_3_<id> (sample counts, unsigned), dimensions
// (neighbour configurations, kernels, densities) with max_k variables.  The
// reference has no job id option and names them with id 4294967295; -id
// sets another.  Flags as in src/auto_qs.cpp:213-336:
//
//   auto_qs_b200 -ti TI -ki K1 [K2 ...] [-maxk 1] [-maxn 80 [N2 ...]] [-nl LIST]
//                [-densities d1 d2 ...] [-maxIter 25000] [-minIter 1000] [-maxT s]
//                [-mpow 2] [-ln 0] [-s SEED] [-id JOB] [-r REPORT] [-W_CUDA 0]
//
// Unsupported options (several TIs, -cti, -fs) stop with a message and status 1.
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
        if (argv[i][0] == '-' && !(argv[i][1] >= '0' && argv[i][1] <= '9') && argv[i][1] != '.') {
            const std::string name = argv[i++];
            bool one = false;
            while (i < argc && !(argv[i][0] == '-' && !(argv[i][1] >= '0' && argv[i][1] <= '9') && argv[i][1] != '.')) {
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

// a flag given once or more (each value after it)
std::vector<std::string> values(const std::multimap<std::string, std::string> &arg, const char *a, const char *b = nullptr) {
    std::vector<std::string> out;
    for (const char *f : {a, b}) {
        if (!f) continue;
        for (auto it = arg.equal_range(f).first; it != arg.equal_range(f).second; ++it)
            if (!it->second.empty()) out.push_back(it->second);
    }
    return out;
}

}  // namespace

int main(int argc, char **argv) {
    auto arg = read_args(argc, argv);
    FILE *rep = stderr;
    if (arg.count("-r") && !arg.find("-r")->second.empty()) {
        FILE *f = std::fopen(arg.find("-r")->second.c_str(), "a");
        if (f) rep = f;
    }
    auto fail = [&](const std::string &msg) {
        std::fprintf(rep, "error: %s\n", msg.c_str());
        if (rep != stderr) std::fclose(rep);
        return 1;
    };
    if (arg.count("-h") || arg.count("--help")) {
        std::printf("auto_qs_b200 -ti TI -ki K1 [K2 ...] [-maxk 1] [-maxn 80 [N2 ...]] [-nl LIST]\n"
                    "             [-densities d1 d2 ...] [-maxIter 25000] [-minIter 1000] [-maxT s] [-mpow 2]\n"
                    "             [-ln 0] [-s SEED] [-id JOB] [-r REPORT] [-W_CUDA DEVICE]\n");
        return 0;
    }
    static const std::set<std::string> known = {"-ti", "-ki", "-maxk", "-maxK", "-maxn", "-maxN", "-nl", "-maxIter",
                                                "-maxiter", "-minIter", "-maxT", "-maxt", "-mpow", "-densities",
                                                "-density", "-ln", "-s", "-id", "-r", "-j", "--jobs", "-W_CUDA",
                                                "-W_GPU", "-v", "--verbose"};
    for (auto &kv : arg)
        if (!known.count(kv.first)) return fail("flag " + kv.first + " is not implemented on the B200 path");
    if (values(arg, "-ti").size() != 1) return fail("exactly one training image (-ti) is supported");
    const auto kernel_names = values(arg, "-ki");
    if (kernel_names.empty()) return fail("no kernel");   // as the reference (src/auto_qs.cpp:317-324)

    Grid ti;
    if (!load(values(arg, "-ti")[0], ti, rep)) return fail("input grids");
    std::vector<Grid> kernels(kernel_names.size());
    std::vector<const float *> kptr;
    std::vector<unsigned> kdims;
    std::vector<int> knvar;
    for (size_t i = 0; i < kernel_names.size(); ++i) {
        if (!load(kernel_names[i], kernels[i], rep)) return fail("kernel grid");
        if (kernels[i].ndim != ti.ndim)
            return fail("kernel " + kernel_names[i] + " must have the training image's dimensions");
        for (int d = 0; d < ti.ndim; ++d) kdims.push_back(kernels[i].dims[d]);
        knvar.push_back(kernels[i].nvar);
        kptr.push_back(kernels[i].data.data());
    }
    const auto num = [&](const char *a, const char *b, double def) {
        const auto v = values(arg, a, b);
        return v.empty() ? def : std::atof(v[0].c_str());
    };
    unsigned max_k = unsigned(num("-maxk", "-maxK", 1));
    std::vector<unsigned> max_n;
    for (auto &v : values(arg, "-maxn", "-maxN")) max_n.push_back(unsigned(std::atoi(v.c_str())));
    std::vector<float> dens;
    for (auto &v : values(arg, "-densities", "-density")) dens.push_back(float(std::atof(v.c_str())));
    if (dens.empty()) dens = {0.0078f, 0.0156f, 0.0312f, 0.0625f, 0.1250f, 0.2500f, 0.5000f};
    // neighbour configurations (src/auto_qs.cpp:650-680)
    std::vector<unsigned> counts;
    int n_counts = 1;
    if (!values(arg, "-nl").empty()) {
        Grid nl;
        if (!load(values(arg, "-nl")[0], nl, rep)) return fail("-nl grid");
        n_counts = nl.nvar;
        for (float x : nl.data) counts.push_back(unsigned(x));
    } else {
        if (max_n.empty()) max_n.push_back(80);
        n_counts = int(max_n.size());
        for (unsigned i = 1; i < max_n[0]; ++i)
            for (unsigned j = 0; j < max_n.size(); ++j) counts.push_back(unsigned(std::round(i * max_n[j] / max_n[0])));
    }
    if (counts.empty()) return fail("no neighbour configuration");
    int device = 0;
    for (const char *w : {"-W_CUDA", "-W_GPU"}) {
        auto v = values(arg, w);
        if (!v.empty()) device = std::atoi(v[0].c_str());
    }
    unsigned seed = values(arg, "-s").empty() ? unsigned(std::chrono::high_resolution_clock::now().time_since_epoch().count())
                                              : unsigned(std::strtoul(values(arg, "-s")[0].c_str(), nullptr, 10));
    const std::string job = values(arg, "-id").empty() ? std::string("4294967295") : values(arg, "-id")[0];

    qsk_calib_params p;
    std::memset(&p, 0, sizeof(p));
    p.ndim = ti.ndim;
    p.ti_dims = ti.dims;
    p.nvar = ti.nvar;
    p.types = ti.types.data();
    p.ti = ti.data.data();
    p.n_kernels = int(kernels.size());
    p.kernel_dims = kdims.data();
    p.kernel_nvar = knvar.data();
    p.kernels = kptr.data();
    p.n_configs = int(counts.size() / size_t(n_counts));
    p.n_counts = n_counts;
    p.counts = counts.data();
    p.n_densities = int(dens.size());
    p.densities = dens.data();
    p.max_k = max_k;
    p.power = float(num("-mpow", nullptr, 2.0));
    p.noise = float(num("-ln", nullptr, 0.0));
    p.max_iterations = unsigned(num("-maxIter", "-maxiter", 25000));
    p.min_iterations = unsigned(num("-minIter", nullptr, 1000));
    p.max_seconds = float(num("-maxT", "-maxt", INFINITY));
    p.seed = seed;
    const size_t n = size_t(p.n_configs) * p.n_kernels * p.n_densities * max_k;
    std::vector<float> mean(n), dev(n);
    std::vector<unsigned> count(n);
    long long searches = 0;
    std::fprintf(rep, "vector calib\n");
    auto t0 = std::chrono::high_resolution_clock::now();
    const int rc = qsk_calibrate(device, &p, mean.data(), dev.data(), count.data(), &searches);
    auto t1 = std::chrono::high_resolution_clock::now();
    if (rc != QSK_OK) return fail(std::string("calibration failed: ") + qsk_last_error());
    const double ms = 1.0e-6 * double(std::chrono::duration_cast<std::chrono::nanoseconds>(t1 - t0).count());
    std::fprintf(rep, "compuattion time: %7.2f s\n", ms / 1000);
    std::fprintf(rep, "compuattion time: %.0f ms\n", ms);
    std::fprintf(rep, "searches: %lld\n", searches);
    // images: (configurations, kernels, densities) x max_k variables
    const unsigned dims[3] = {unsigned(p.n_configs), unsigned(p.n_kernels), unsigned(p.n_densities)};
    std::vector<int> types(max_k, 0);
    const std::string dir = data_dir() + "/";
    if (qsk_bgrid_write((dir + "im_3_" + job + ".bgrid").c_str(), 3, dims, int(max_k), types.data(), 2, count.data(), 0) ||
        qsk_bgrid_write((dir + "im_2_" + job + ".bgrid").c_str(), 3, dims, int(max_k), types.data(), 0, dev.data(), 0) ||
        qsk_bgrid_write((dir + "im_1_" + job + ".bgrid").c_str(), 3, dims, int(max_k), types.data(), 0, mean.data(), 0))
        return fail(qsk_last_error());
    if (rep != stderr) std::fclose(rep);
    return 0;
}
