// C ABI of the learned sizer (include/partc.h): create / load / save / train / predict.
#include <chrono>
#include <cstdio>
#include <cstring>
#include <string>

#include "partc.h"
#include "ptc_sizer.cuh"

namespace ptc {

namespace {

constexpr char kMagic[8] = {'P', 'T', 'C', 'S', 'Z', 'R', '0', '1'};
constexpr int kMaxStreamDevices = 64;

cudaStream_t sizer_stream(int32_t device) {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        throw Error{PTC_ERR_NO_DEVICE, "no usable CUDA device"};
    }
    if (device >= 0) PTC_CUDA(cudaSetDevice(device));
    int cur = 0;
    PTC_CUDA(cudaGetDevice(&cur));
    PTC_REQUIRE(cur < kMaxStreamDevices, PTC_ERR_INVALID_ARGUMENT, "device ordinal out of range");
    // one stream per device and host thread, kept for the thread's lifetime
    thread_local cudaStream_t streams[kMaxStreamDevices] = {};
    if (!streams[cur]) PTC_CUDA(cudaStreamCreateWithFlags(&streams[cur], cudaStreamNonBlocking));
    return streams[cur];
}

template <typename F>
ptc_status guarded(F&& f) {
    DeviceGuard keep_device;
    try {
        f();
        return PTC_OK;
    } catch (const Error& e) {
        set_last_error(e.status, e.msg);
        return e.status;
    } catch (const std::bad_alloc&) {
        set_last_error(PTC_ERR_OUT_OF_MEMORY, "host allocation failed");
        return PTC_ERR_OUT_OF_MEMORY;
    } catch (...) {
        set_last_error(PTC_ERR_INTERNAL, "unexpected exception");
        return PTC_ERR_INTERNAL;
    }
}

float* to_device(Arena& ar, const float* h, uint64_t n) {
    float* d = ar.alloc<float>(n);
    PTC_CUDA(cudaMemcpyAsync(d, h, n * sizeof(float), cudaMemcpyHostToDevice, ar.stream()));
    return d;
}

}  // namespace

}  // namespace ptc

using ptc::Error;

extern "C" {

void ptc_train_options_init(ptc_train_options* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->struct_size = sizeof(*o);
    o->epochs = 20;
    o->batch = 8192;
    o->lr = 2e-3f;
    o->seed = 7;
    o->device = -1;
}

ptc_status ptc_sizer_create(uint64_t seed, ptc_sizer** out) {
    return ptc::guarded([&] {
        PTC_REQUIRE(out != nullptr, PTC_ERR_INVALID_ARGUMENT, "out is null");
        auto* s = new ptc_sizer;
        ptc::sizer_init(s->host, seed);
        *out = s;
    });
}

void ptc_sizer_free(ptc_sizer* s) { delete s; }

ptc_status ptc_sizer_get_params(const ptc_sizer* s, float* params) {
    return ptc::guarded([&] {
        PTC_REQUIRE(s && params, PTC_ERR_INVALID_ARGUMENT, "null argument");
        std::memcpy(params, s->host.master.data(), ptc::kSizerParams * sizeof(float));
    });
}

ptc_status ptc_sizer_set_params(ptc_sizer* s, const float* params) {
    return ptc::guarded([&] {
        PTC_REQUIRE(s && params, PTC_ERR_INVALID_ARGUMENT, "null argument");
        std::memcpy(s->host.master.data(), params, ptc::kSizerParams * sizeof(float));
    });
}

ptc_status ptc_sizer_save(const ptc_sizer* s, const char* path) {
    return ptc::guarded([&] {
        PTC_REQUIRE(s && path, PTC_ERR_INVALID_ARGUMENT, "null argument");
        FILE* f = std::fopen(path, "wb");
        PTC_REQUIRE(f != nullptr, PTC_ERR_INVALID_ARGUMENT, std::string("cannot write ") + path);
        const uint32_t n = ptc::kSizerParams;
        const bool ok = std::fwrite(ptc::kMagic, 1, 8, f) == 8 && std::fwrite(&n, 4, 1, f) == 1 &&
                        std::fwrite(s->host.master.data(), sizeof(float), n, f) == n;
        std::fclose(f);
        PTC_REQUIRE(ok, PTC_ERR_INVALID_ARGUMENT, std::string("short write to ") + path);
    });
}

ptc_status ptc_sizer_load(const char* path, ptc_sizer** out) {
    return ptc::guarded([&] {
        PTC_REQUIRE(path && out, PTC_ERR_INVALID_ARGUMENT, "null argument");
        FILE* f = std::fopen(path, "rb");
        PTC_REQUIRE(f != nullptr, PTC_ERR_INVALID_ARGUMENT, std::string("cannot read ") + path);
        char magic[8];
        uint32_t n = 0;
        auto* s = new ptc_sizer;
        ptc::sizer_init(s->host, 0);
        const bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, ptc::kMagic, 8) == 0 &&
                        std::fread(&n, 4, 1, f) == 1 && n == (uint32_t)ptc::kSizerParams &&
                        std::fread(s->host.master.data(), sizeof(float), n, f) == n;
        std::fclose(f);
        if (!ok) {
            delete s;
            throw Error{PTC_ERR_INVALID_ARGUMENT, std::string("not a sizer weight file: ") + path};
        }
        *out = s;
    });
}

ptc_status ptc_sizer_train(ptc_sizer* s, const float* features, const float* targets, uint64_t n,
                           const ptc_train_options* opt_in, ptc_train_stats* stats) {
    return ptc::guarded([&] {
        PTC_REQUIRE(s && features && targets, PTC_ERR_INVALID_ARGUMENT, "null argument");
        PTC_REQUIRE(n < (1ull << 32), PTC_ERR_INVALID_ARGUMENT, "too many samples");
        ptc_train_options opt;
        ptc_train_options_init(&opt);
        if (opt_in) std::memcpy(&opt, opt_in, std::min<size_t>(opt_in->struct_size, sizeof(opt)));
        const auto t0 = std::chrono::steady_clock::now();
        cudaStream_t st = ptc::sizer_stream(opt.device);
        ptc::Arena ar(st);
        float* dx = ptc::to_device(ar, features, n * ptc::kSizerInputs);
        float* dt = ptc::to_device(ar, targets, n);
        const ptc::SizerTrainResult r =
            ptc::sizer_train(s->host, dx, dt, n, opt.epochs, opt.batch, opt.lr, opt.seed, ar);
        ar.release();
        PTC_CUDA(cudaStreamSynchronize(st));
        if (stats) {
            stats->first_epoch_loss = r.first_loss;
            stats->final_epoch_loss = r.final_loss;
            stats->epochs = r.epochs;
            stats->steps = r.steps;
            stats->ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        }
    });
}

ptc_status ptc_sizer_predict(const ptc_sizer* s, const float* features, uint64_t n, int32_t device, float* out) {
    return ptc::guarded([&] {
        PTC_REQUIRE(s && features && out, PTC_ERR_INVALID_ARGUMENT, "null argument");
        cudaStream_t st = ptc::sizer_stream(device);
        ptc::Arena ar(st);
        float* dx = ptc::to_device(ar, features, n * ptc::kSizerInputs);
        float* dy = ar.alloc<float>(n);
        ptc::sizer_predict_device(s->host, dx, n, dy, ar);
        PTC_CUDA(cudaMemcpyAsync(out, dy, n * sizeof(float), cudaMemcpyDeviceToHost, st));
        ar.release();
        PTC_CUDA(cudaStreamSynchronize(st));
    });
}

ptc_status ptc_sizer_gradients(const ptc_sizer* s, const float* features, const float* targets, uint64_t n,
                               int32_t device, float* grads, float* loss) {
    return ptc::guarded([&] {
        PTC_REQUIRE(s && features && targets && grads && n > 0, PTC_ERR_INVALID_ARGUMENT, "bad argument");
        cudaStream_t st = ptc::sizer_stream(device);
        ptc::Arena ar(st);
        float* dx = ptc::to_device(ar, features, n * ptc::kSizerInputs);
        float* dt = ptc::to_device(ar, targets, n);
        const float l = ptc::sizer_gradients(s->host, dx, dt, n, grads, ar);
        if (loss) *loss = l;
        ar.release();
        PTC_CUDA(cudaStreamSynchronize(st));
    });
}

void ptc_buffer_free(void* p) { std::free(p); }

}  // extern "C"
