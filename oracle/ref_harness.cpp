/*
 * Test infrastructure only — drives the G2S reference QuickSampling (compiled
 * from the G2S sources by oracle/Makefile, never copied here) in-process, so
 * that tests and the CPU-baseline leg of bench.py can run the unmodified
 * reference CPU path on the same synthetic inputs as the GPU path.
 *
 * Wraps: g2s::DataImage serialisation (G2S include/DataImage.hpp:143-168,
 * 281-320, src/DataImage.cpp:101-165) and g2sQsProgramMain (G2S
 * src/qs.cpp:364), which reads/writes /tmp/G2S/data/<name>.bgrid[.gz].
 */
#include <sys/stat.h>
#include <cstring>
#include <string>
#include <vector>

#include "DataImage.hpp"
#include "qsCore.hpp"

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

}
