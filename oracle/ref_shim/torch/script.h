/*
 * torch/script.h -- minimal stand-in for the libtorch calls the reference's
 * boundary-net code makes (mesh.cpp:2778-2819 and siblings), used only to
 * compile the reference sources as a test checker.  torch::jit::load maps the
 * archive's file name (AutoT0x.pt) to raw float32 weights AutoT0x.f32 in the
 * directory named by IPPI_REF_NN_DIR (TorchScript parameter order); the
 * forward pass is the oracle's float32 restatement of the Net (Linear+ReLU x7,
 * Linear).  A missing weight file gives a module whose output is 0, which the
 * reference treats as "no learned tau" (NNflag = false, Smagorinsky tau).
 */
#ifndef IPPI_REF_TORCH_SHIM_H
#define IPPI_REF_TORCH_SHIM_H
#include <cstdio>
#include <cstdlib>
#include <initializer_list>
#include <memory>
#include <string>
#include <vector>

extern "C" float orc_band_forward(const float* w, int nin, const float* in);

namespace torch {
enum DeviceType { kCPU = 0 };
enum ScalarType { kFloat32 = 0, kFloat = 0 };
struct Device {
    Device(DeviceType) {}
};
struct NoGradGuard {};
struct Tensor {
    std::vector<float> v;
    Tensor reshape(std::initializer_list<long>) const { return *this; }
    Tensor to(const Device&) const { return *this; }
    template <typename T> T item() const { return (T)v.at(0); }
};
inline Tensor from_blob(void* p, std::initializer_list<long> shape, ScalarType)
{
    long n = 1;
    for (long s : shape) n *= s;
    Tensor t;
    t.v.assign((const float*)p, (const float*)p + n);
    return t;
}
namespace jit {
struct IValue {
    Tensor t;
    IValue(const Tensor& x) : t(x) {}
    Tensor toTensor() const { return t; }
};
namespace script {
struct Module {
    std::shared_ptr<std::vector<float>> w;
    IValue forward(const std::vector<IValue>& in)
    {
        Tensor out;
        const std::vector<float>& x = in.at(0).t.v;
        float y = 0.f;
        if (w && !w->empty()) y = orc_band_forward(w->data(), (int)x.size(), x.data());
        out.v.assign(1, y);
        return IValue(out);
    }
};
}  // namespace script
using script::Module;
inline script::Module load(const std::string& path, const Device&)
{
    script::Module m;
    const char* dir = std::getenv("IPPI_REF_NN_DIR");
    if (!dir) return m;
    std::string base = path.substr(path.find_last_of('/') + 1);
    std::string stem = base.substr(0, base.find_last_of('.'));
    std::string f = std::string(dir) + "/" + stem + ".f32";
    FILE* fp = std::fopen(f.c_str(), "rb");
    if (!fp) return m;
    m.w = std::make_shared<std::vector<float>>();
    float buf[4096];
    size_t r;
    while ((r = std::fread(buf, sizeof(float), 4096, fp)) > 0) m.w->insert(m.w->end(), buf, buf + r);
    std::fclose(fp);
    return m;
}
}  // namespace jit
}  // namespace torch
#endif
