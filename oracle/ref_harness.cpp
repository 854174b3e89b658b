/*
 * Test infrastructure only — drives the G2S reference QuickSampling (compiled
 * from the G2S sources by oracle/Makefile, never copied here) in-process, so
 * that tests and the CPU-baseline leg of bench.py can run the unmodified
 * reference CPU path on the same synthetic inputs as the GPU path.
 *
 * Wraps: g2s::DataImage serialisation (G2S include/DataImage.hpp:143-168,
 * 281-320, src/DataImage.cpp:101-165), g2sQsProgramMain (G2S
 * src/qs.cpp:364), which reads/writes /tmp/G2S/data/<name>.bgrid[.gz], and
 * QuantileSamplingModule::distribution on a CPU device set up the way
 * src/auto_qs.cpp:531-640 sets up its calibration module (the auto_qs
 * calibration's per-sample search, include/calibration.hpp:221-224).
 */
#include <sys/stat.h>
#include <cstring>
#include <string>
#include <vector>

#include "CPUThreadDevice.hpp"
#include "DataImage.hpp"
#include "qsCore.hpp"
#include "quantileSamplingModule.hpp"
#include "sharedMemoryManager.hpp"

extern "C" {

/* Write a grid (x fastest, variables interleaved) as /tmp/G2S/data/<name>.bgrid.
 * types[v]: 0 continuous, 1 categorical. Returns 0 on success. */
int g2sref_write_image(const char *name, int ndim, const unsigned *dims, int nvar, const int *types,
                       const float *data, int compressed) {
    (void)mkdir("/tmp/G2S", 0770);
    (void)mkdir("/tmp/G2S/data", 0770);
    (void)mkdir("/tmp/G2S/logs", 0770);
    std::vector<unsigned> d(dims, dims + ndim);
    g2s::DataImage image(unsigned(ndim), d.data(), unsigned(nvar));
    for (int v = 0; v < nvar; ++v)
        image._types[v] = types[v] == 1 ? g2s::DataImage::Categorical : g2s::DataImage::Continuous;
    std::memcpy(image._data, data, sizeof(float) * image.dataSize());
    image.write(std::string(name), compressed != 0);
    return 0;
}

/* Read /tmp/G2S/data/<name>.bgrid[.gz].  dims must hold 16 entries.  Returns
 * the number of floats available (copies at most cap), or -1. */
long g2sref_read_image(const char *name, int *ndim, unsigned *dims, int *nvar, int *encoding, float *data,
                       long cap) {
    g2s::DataImage image = g2s::DataImage::createFromFile(std::string(name));
    if (image.isEmpty()) return -1;
    *ndim = int(image._dims.size());
    for (size_t i = 0; i < image._dims.size() && i < 16; ++i) dims[i] = image._dims[i];
    *nvar = int(image._nbVariable);
    *encoding = int(image._encodingType);
    long n = long(image.dataSize());
    if (data) std::memcpy(data, image._data, sizeof(float) * size_t(n < cap ? n : cap));
    return n;
}

/* Run the reference qs program with argv (argv[0] is the program name). */
int g2sref_qs_main(int argc, const char **argv) { return g2sQsProgramMain(argc, argv); }

/* One QuantileSamplingModule::distribution query on one complete TI (x
 * fastest, variables interleaved, types 0/1) with a weight kernel (kdims,
 * knvar variables): nnb neighbour offsets and values (NaN: absent), k
 * candidates, seed, the origin TI cell and the verbatim radius.  Writes the
 * k TI positions in the order distribution() returns them.  Returns 0. */
int g2sref_distribution(int nd, const unsigned *dims, int nvar, const int *types, const float *ti,
                        const unsigned *kdims, int knvar, const float *kernel, int nnb, const int *offs,
                        const float *vals, unsigned k, float seed, unsigned origin, float radius,
                        unsigned *out_position) {
    std::vector<unsigned> d(dims, dims + nd), kd(kdims, kdims + nd);
    g2s::DataImage image(unsigned(nd), d.data(), unsigned(nvar));
    for (int v = 0; v < nvar; ++v)
        image._types[v] = types[v] == 1 ? g2s::DataImage::Categorical : g2s::DataImage::Continuous;
    std::memcpy(image._data, ti, sizeof(float) * image.dataSize());
    g2s::DataImage kimage(unsigned(nd), kd.data(), unsigned(knvar));
    std::memcpy(kimage._data, kernel, sizeof(float) * kimage.dataSize());

    // categories in order of first appearance, one indicator variable each
    std::vector<std::vector<float> > categories;
    std::vector<unsigned> perVariable;
    for (int v = 0; v < nvar; ++v) {
        if (types[v] != 1) {
            perVariable.push_back(1);
            continue;
        }
        std::vector<float> cv;
        for (size_t j = size_t(v); j < image.dataSize(); j += size_t(nvar)) {
            const float x = image._data[j];
            if (std::isnan(x)) continue;
            bool seen = false;
            for (float c : cv) seen |= (c == x);
            if (!seen) cv.push_back(x);
        }
        categories.push_back(cv);
        perVariable.push_back(unsigned(cv.size()));
    }
    g2s::DataImage kexp = g2s::DataImage::offsetKernel4categories(kimage, perVariable);

    std::vector<g2s::OperationMatrix> coef;
    std::vector<std::vector<conversionType> > convMain;
    std::vector<std::vector<std::vector<conversionType> > > convConst;
    std::vector<std::vector<std::vector<float> > > coefConst;
    image.generateCoefMatrix4Xcorr(coef, convMain, convConst, coefConst, false, categories);
    SharedMemoryManager *smm = new SharedMemoryManager(image._dims);
    std::vector<std::vector<g2s::DataImage> > layers = image.convertInput4Xcorr(smm->_fftSize, false, categories);
    for (auto &group : layers)
        for (auto &layer : group) smm->addVariable(layer._data);
    std::vector<ComputeDeviceModule *> *devices = new std::vector<ComputeDeviceModule *>[1];
    CPUThreadDevice *cpu = new CPUThreadDevice(smm, coef, 1, false, false);
    cpu->setTrueMismatch(false);
    devices[0].push_back(cpu);
    smm->allowNewModule(false);
    {
        QuantileSamplingModule qsm(devices, nullptr, float(k), convMain, convConst, coefConst, true, true, 1, 1, 1,
                                   false);
        // neighbours in the module's variable layout (categories as indicators)
        std::vector<std::vector<int> > nbOffsets;
        std::vector<std::vector<float> > nbValues;
        for (int j = 0; j < nnb; ++j) {
            nbOffsets.push_back(std::vector<int>(offs + j * nd, offs + (j + 1) * nd));
            std::vector<float> row;
            unsigned c = 0;
            for (int v = 0; v < nvar; ++v) {
                const float x = vals[j * nvar + v];
                if (types[v] != 1) {
                    row.push_back(x);
                    continue;
                }
                for (float cat : categories[c]) row.push_back(x == cat ? 1.f : 0.f);
                c++;
            }
            nbValues.push_back(row);
        }
        SamplingModule::matchLocation o;
        o.TI = 0;
        o.index = origin;
        std::vector<SamplingModule::matchLocation> res =
            qsm.distribution(nbOffsets, nbValues, seed, o, radius, 0, false, 0, 0.f, -1, &kexp);
        for (unsigned i = 0; i < k && i < res.size(); ++i) out_position[i] = res[i].index;
    }
    delete cpu;
    delete[] devices;
    delete smm;
    return 0;
}

}
