// Drop-in accelerator device for G2S `qs -W_CUDA`: the two symbols that
// G2S src/qs.cpp:861-911 resolves from dlopen("./g2s_cuda.so"), implemented
// on the B200 C ABI of libg2s_b200.so (include/g2s_b200.h).
//
// This file is compiled against the G2S headers (AcceleratorDevice.hpp and
// its includes), because the object it returns must be a G2S
// AcceleratorDevice: QuantileSamplingModule drives it through that class's
// virtual interface (include/AcceleratorDevice.hpp:37-91).  Every
// per-node computation goes to the GPU; nothing here computes a map.
//
// Behaviour:
//  * allocAndInitSharedMemory uploads the correlation layers once per GPU and
//    hands the qsk_ti handle to the other devices on that GPU through the
//    SharedMemoryManager address slots (src/sharedMemoryManager.cpp:72-125).
//  * candidateForPattern (overridden: map + border in one pass) records the
//    pattern as terms "coefficient x layer at neighbour" in the reference's
//    layer decomposition (CPUThreadDevice.cpp:386-446);
//  * searchKBiggest runs the fused map + k-best on the GPU with the CPU
//    path's tie-breaking (fKb.hpp) and returns scores scaled like the device
//    that qs asked for (setTrueMismatch(true): S/N·N + delta, i.e. S + delta;
//    otherwise the unnormalised N·S of the CPU device);
//  * training images with missing values: the overlap ("cross") output of the
//    XMeasurement matrix, its centre mask and the -|S/c^4| compensation are
//    applied on the GPU (qsk_pattern_opts); -nV excludes one candidate, or,
//    with a verbatim radius (auto_qs' distribution() queries), every index
//    that the CPU device's setValueInErrorArrayWithRadius marks
//    (CPUThreadDevice.cpp:310-342; the reference CUDA device leaves that
//    method empty, NvidiaGPUAcceleratorDevice.cu:646-670).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <vector>

#include "AcceleratorDevice.hpp"
#include "sharedMemoryManager.hpp"
#include "g2s_b200.h"

namespace {

void check(int rc, const char *what) {
    if (rc != QSK_OK) {
        char buf[768];
        snprintf(buf, sizeof(buf), "g2s_b200: %s failed (%d): %s", what, rc, qsk_last_error());
        fprintf(stderr, "%s\n", buf);
        throw std::runtime_error(buf);
    }
}

class B200QsDevice : public AcceleratorDevice {
public:
    B200QsDevice(int deviceId, SharedMemoryManager *smm, std::vector<g2s::OperationMatrix> coefficientMatrix,
                 unsigned threadRatio, bool withCrossMeasurement, bool circularTI)
        : AcceleratorDevice(smm, coefficientMatrix, threadRatio, withCrossMeasurement, circularTI) {
        if (circularTI) throw std::runtime_error("g2s_b200: circular training images are not supported");
        _deviceType = DT_gpuCuda;
        _deviceID = unsigned(deviceId);
        _gpu = deviceId;
#pragma omp critical(createDevices)
        { _sharedMemoryManager->addDevice(this); }
        initDim();
        _ti = static_cast<qsk_ti *>(_srcCplx.at(0).fft);
        check(qsk_worker_create(_ti, &_worker), "qsk_worker_create");
    }

    ~B200QsDevice() {
        if (_worker) qsk_worker_destroy(_worker);
        _sharedMemoryManager->removeDevice(this);
    }

    std::vector<g2s::spaceFrequencyMemoryAddress> allocAndInitSharedMemory(std::vector<void *> srcMemoryAddress,
                                                                           std::vector<unsigned> srcSize,
                                                                           std::vector<unsigned> fftSize) override {
        std::vector<const float *> layers;
        for (void *p : srcMemoryAddress) layers.push_back(static_cast<const float *>(p));
        qsk_ti *ti = nullptr;
        check(qsk_ti_create_layers(_gpu, int(srcSize.size()), srcSize.data(), fftSize.data(), int(layers.size()),
                                   layers.data(), &ti),
              "qsk_ti_create_layers");
        std::vector<g2s::spaceFrequencyMemoryAddress> out(srcMemoryAddress.size());
        for (auto &a : out) {
            a.space = nullptr;
            a.fft = ti;   // every device on this GPU finds the shared TI here
        }
        return out;
    }

    std::vector<g2s::spaceFrequencyMemoryAddress> freeSharedMemory(
        std::vector<g2s::spaceFrequencyMemoryAddress> sharedMemoryAddress) override {
        if (!sharedMemoryAddress.empty()) qsk_ti_destroy(static_cast<qsk_ti *>(sharedMemoryAddress[0].fft));
        sharedMemoryAddress.clear();
        return sharedMemoryAddress;
    }

    bool candidateForPattern(std::vector<std::vector<int>> &neighborArrayVector,
                             std::vector<std::vector<float>> &neighborValueArrayVector, std::vector<float> &,
                             std::vector<float> delta0) override {
        if (neighborValueArrayVector.size() == 0) return false;
        const int nd = int(_fftSize.size());
        for (int d = 0; d < nd; ++d) _min[d] = _max[d] = 0;
        _offsets.clear();
        for (auto &o : neighborArrayVector)
            for (int d = 0; d < nd; ++d) {
                _offsets.push_back(o[d]);
                _min[d] = std::min(_min[d], o[d]);
                _max[d] = std::max(_max[d], o[d]);
            }
        // terms: neighbour j, its converted value var, every layer varA with a
        // non-zero coefficient in the regular operation matrix; with missing
        // training-image values also the overlap terms of the XMeasurement
        // matrix (DataImage.hpp:626-710, CPUThreadDevice.cpp:426-444)
        g2s::OperationMatrix &M = _coefficientMatrix[0];
        const int nvar = int(M.getNumberOfVariable());
        _terms.clear();
        for (size_t j = 0; j < neighborValueArrayVector.size(); ++j) {
            const std::vector<float> &vals = neighborValueArrayVector[j];
            for (int var = 0; var < nvar && var < int(vals.size()); ++var) {
                if (std::isnan(vals[var])) continue;
                for (size_t mi = 0; mi < _coefficientMatrix.size() && mi < 2; ++mi) {
                    g2s::OperationMatrix &Mi = _coefficientMatrix[mi];
                    for (int varA = 0; varA < nvar; ++varA) {
                        float c = Mi.getVariableAt(varA, var);
                        if (c == 0.f) continue;
                        float coef = c * vals[var];
                        if (coef == 0.f) continue;
                        qsk_term t;
                        t.neighbour = int(j);
                        t.layer = varA;
                        t.op = mi == 0 ? QSK_OP_LIN : QSK_OP_LIN_CROSS;
                        t.a = coef;
                        t.b = 0.f;
                        _terms.push_back(t);
                    }
                }
            }
        }
        _opts.exclude_index = -1;
        _opts.exclude_radius = 0.f;
        _opts.missing_data = 0;
        _opts.centre_mask_layer = -1;
        _delta = delta0.empty() ? 0.f : delta0[0];
        _nnb = int(neighborArrayVector.size());
        return true;
    }

    void searchKBiggest(float *errors, unsigned *encodedPosition, unsigned extendK, float seed) override {
        std::vector<int> mn(_fftSize.size());
        check(qsk_pattern_kbest_ex(_worker, _nnb, _offsets.data(), int(_terms.size()), _terms.data(), extendK, seed,
                                   &_opts, errors, encodedPosition, mn.data()),
              "qsk_pattern_kbest_ex");
        if (!_opts.missing_data) {
            // the reference CUDA device reports S + delta, the CPU device N*S
            const float N = float(_realSpaceSize);
            for (unsigned j = 0; j < extendK; ++j) errors[j] = _trueMismatch ? errors[j] + _delta : errors[j] * N;
        }
        _opts.exclude_index = -1;
        _opts.exclude_radius = 0.f;
    }

    unsigned getErrorsArraySize() override { return _realSpaceSize; }
    unsigned getArraySize() override { return _realSpaceSize; }
    float getErrorAtPosition(unsigned) override { return NAN; }
    float getValueAtPosition(unsigned, unsigned) override { return NAN; }
    float getCrossErrorAtPosition(unsigned) override { return NAN; }

    unsigned cvtIndexToPosition(unsigned index) override { return qsk_index_to_position(_ti, _min.data(), index); }
    unsigned cvtPositionToIndex(unsigned position) override {
        return qsk_position_to_index(_ti, _min.data(), position);
    }

    // cross output masked by the TI mask at the candidate centre
    // (CPUThreadDevice.cpp:501-524): the mask layer is the first layer with a
    // non-zero row in the XMeasurement matrix
    void maskLayerWithVariable(unsigned, unsigned variable) override {
        if (_coefficientMatrix.size() < 2) throw std::runtime_error("g2s_b200: no cross-measurement matrix");
        g2s::OperationMatrix &X = _coefficientMatrix[1];
        int tmp = int(variable), conv = 0;
        for (unsigned var = 0; var < X.getNumberOfVariable(); ++var) {
            tmp -= X.needVariableAlongA(int(var));
            if (tmp < 0) {
                conv = int(var);
                break;
            }
        }
        _opts.centre_mask_layer = conv;
    }
    // -nV: the excluded candidate (quantileSamplingModule.hpp:566-571); the
    // reference only ever writes -inf here
    void setValueInErrorArray(unsigned position, float) override {
        _opts.exclude_index = int(position);
        _opts.exclude_radius = 0.f;
    }
    void setValueInErrorArrayWithRadius(unsigned position, float, float radius) override {
        _opts.exclude_index = int(position);
        _opts.exclude_radius = radius;
    }
    // -|S / c^4|, -inf where c == 0 (NvidiaGPUAcceleratorDevice.cu:199-206,677-686)
    void compensateMissingData() override { _opts.missing_data = 1; }

    // the FFT pipeline steps are replaced by the fused candidateForPattern
    void zerosFrenquencySpaceOutputArray(unsigned) override {}
    void computeFreqMismatchMap(std::vector<std::vector<int>>, std::vector<std::vector<float>> &) override {}
    void computeRealMissmatchAndRemoveWrongPattern(float *) override {}

private:
    int _gpu = 0;
    qsk_ti *_ti = nullptr;
    qsk_worker *_worker = nullptr;
    std::vector<int> _offsets;
    std::vector<qsk_term> _terms;
    qsk_pattern_opts _opts{-1, 0, -1, 0.f};
    int _nnb = 0;
    float _delta = 0.f;
};

}  // namespace

extern "C" {

// G2S src/NvidiaGPUAcceleratorDevice.cu:26-30
void g2s_cudaGetDeviceCount(int *count) {
    if (qsk_device_count(count) != QSK_OK) *count = 0;
}

// G2S src/NvidiaGPUAcceleratorDevice.cu:229-233 (typedef src/qs.cpp:865)
AcceleratorDevice *c_NvidiaGPUAcceleratorDevice(int deviceId, SharedMemoryManager *sharedMemoryManager,
                                                std::vector<g2s::OperationMatrix> coefficientMatrix,
                                                unsigned int threadRatio, bool withCrossMeasurement, bool circularTI) {
    return new B200QsDevice(deviceId, sharedMemoryManager, coefficientMatrix, threadRatio, withCrossMeasurement,
                            circularTI);
}

}
