// ippi_autograd.cpp -- libtorch torch::autograd::Function wrappers of a
// solver rollout, over the C ABI of libippi_lbm.so (include/ippi_lbm.h).
//
// A rollout is nsteps steps of a lattice from a fixed starting state.  The
// forward pass restores that state (ippi_load_state), applies the parameters
// being differentiated (a tau field, or the learned network's FP32
// weights), and runs the checkpointed forward (ippi_adjoint_forward: one
// population buffer kept every ckpt_every steps).  It returns the body force
// of every step [nsteps][nbody][2] and the last step's post-stream rho, ux,
// uy [3][ny][nx], FP64 on the CPU.  The backward pass is the library's
// hand-written adjoint (ippi_adjoint_backward: each segment recomputed from
// its checkpoint, then the reverse sweep), which returns the gradient with
// respect to the parameters.  torch carries the tensors; every derivative
// comes from the library.
//
// The starting state is captured when the rollout object is made, from the
// lattice as the caller left it (after its initial fields and any warm-up
// steps), together with the parameters in force then ("base"): a checkpoint
// presumes the tau field or network it was taken under, so every forward
// pass puts the base parameters back before it restores the state.
#include <torch/extension.h>

#include <stdexcept>
#include <string>
#include <vector>

#include "ippi_lbm.h"

namespace ippi_torch {

using torch::Tensor;
using torch::autograd::AutogradContext;
using torch::autograd::variable_list;

void check(ippi_lbm* h, int rc, const char* what)
{
    if (rc == IPPI_OK) return;
    char buf[512];
    ippi_last_error(h, buf, sizeof buf);
    throw std::runtime_error(std::string(what) + ": ippi error " + std::to_string(rc) + ": " + buf);
}

// the parameters a rollout differentiates
enum class Param { TauField, Network };

struct Rollout {
    ippi_lbm* h = nullptr;
    Param kind = Param::TauField;
    int nx = 0, ny = 0, nbody = 0;
    int nsteps = 0, t0 = 1, ckpt = 64;
    std::vector<unsigned char> state;  // ippi_save_state of the starting point
    std::vector<double> base_tau;      // [ny][nx] (TauField)
    std::vector<float> base_w, stats;  // [1313], [25] (Network)

    void apply(const Tensor& p) const
    {
        if (kind == Param::TauField) {
            Tensor t = p.detach().to(torch::kCPU, torch::kFloat64).contiguous();
            TORCH_CHECK(t.numel() == (int64_t)nx * ny, "tau field needs ", (int64_t)nx * ny, " values");
            check(h, ippi_set_tau_field(h, t.data_ptr<double>()), "ippi_set_tau_field");
        } else {
            Tensor w = p.detach().to(torch::kCPU, torch::kFloat32).contiguous();
            TORCH_CHECK(w.numel() == IPPI_MLP_PARAMS, "network needs ", IPPI_MLP_PARAMS, " weights");
            check(h, ippi_load_tau_mlp_f32(h, w.data_ptr<float>(), IPPI_MLP_PARAMS, stats.data(), stats.size()),
                  "ippi_load_tau_mlp_f32");
        }
    }

    void restore_base() const
    {
        if (kind == Param::TauField)
            check(h, ippi_set_tau_field(h, base_tau.data()), "ippi_set_tau_field");
        else
            check(h, ippi_load_tau_mlp_f32(h, base_w.data(), IPPI_MLP_PARAMS, stats.data(), stats.size()),
                  "ippi_load_tau_mlp_f32");
        check(h, ippi_load_state(h, state.data(), state.size(), nullptr), "ippi_load_state");
    }

    // forward pass: (forces [nsteps][nbody][2], macros [3][ny][nx])
    std::pair<Tensor, Tensor> run(const Tensor& p) const
    {
        restore_base();
        apply(p);
        check(h, ippi_adjoint_forward(h, nsteps, t0, ckpt), "ippi_adjoint_forward");
        auto opt = torch::TensorOptions().dtype(torch::kFloat64);
        Tensor forces = torch::zeros({nsteps, std::max(nbody, 1), 2}, opt);
        if (nbody > 0) {
            const int got = ippi_force_history(h, forces.data_ptr<double>(), nsteps);
            if (got < 0) check(h, got, "ippi_force_history");
            TORCH_CHECK(got == nsteps, "force history holds ", got, " of ", nsteps, " steps");
        }
        forces = forces.narrow(1, 0, nbody);
        Tensor macros = torch::empty({3, ny, nx}, opt);
        const size_t plane = (size_t)nx * ny * sizeof(double);
        const int fields[3] = {IPPI_FIELD_RHO, IPPI_FIELD_UX, IPPI_FIELD_UY};
        for (int q = 0; q < 3; q++)
            check(h, ippi_download(h, fields[q], macros.data_ptr<double>() + (size_t)q * nx * ny, plane),
                  "ippi_download");
        return {forces, macros};
    }

    Tensor grad(const Tensor& g_forces, const Tensor& g_macros) const
    {
        Tensor dF, dM;
        const double* pF = nullptr;
        const double* pM = nullptr;
        if (g_forces.defined() && nbody > 0) {
            dF = g_forces.detach().to(torch::kCPU, torch::kFloat64).contiguous();
            pF = dF.data_ptr<double>();
        }
        if (g_macros.defined()) {
            dM = g_macros.detach().to(torch::kCPU, torch::kFloat64).contiguous();
            pM = dM.data_ptr<double>();
        }
        auto opt = torch::TensorOptions().dtype(torch::kFloat64);
        if (kind == Param::TauField) {
            Tensor g = torch::zeros({ny, nx}, opt);
            check(h, ippi_adjoint_backward(h, pF, pM, g.data_ptr<double>(), nullptr, nullptr),
                  "ippi_adjoint_backward");
            return g;
        }
        Tensor g = torch::zeros({IPPI_MLP_PARAMS}, opt);
        check(h, ippi_adjoint_backward(h, pF, pM, nullptr, g.data_ptr<double>(), nullptr), "ippi_adjoint_backward");
        return g;
    }
};

// the rollout as a TorchScript custom class, so the autograd context can hold
// a reference to it until the backward pass has run
struct RolloutHolder : torch::CustomClassHolder {
    Rollout r;
};

c10::intrusive_ptr<RolloutHolder> make_rollout(int64_t handle, Param kind, int64_t nsteps, int64_t t0,
                                               int64_t ckpt, const Tensor& base, const Tensor& stats,
                                               int64_t nx = 0, int64_t ny = 0)
{
    auto hold = c10::make_intrusive<RolloutHolder>();
    Rollout& r = hold->r;
    r.h = reinterpret_cast<ippi_lbm*>(static_cast<intptr_t>(handle));
    TORCH_CHECK(r.h, "null lattice handle");
    TORCH_CHECK(nsteps > 0 && ckpt > 0, "nsteps and ckpt_every must be positive");
    r.kind = kind;
    r.nsteps = (int)nsteps;
    r.t0 = (int)t0;
    r.ckpt = (int)ckpt;
    int nb = 0;
    check(r.h, ippi_forces(r.h, nullptr, &nb, nullptr), "ippi_forces");
    r.nbody = nb;
    size_t bytes = 0;
    check(r.h, ippi_state_bytes(r.h, &bytes), "ippi_state_bytes");
    r.state.resize(bytes);
    check(r.h, ippi_save_state(r.h, r.state.data(), bytes), "ippi_save_state");
    if (kind == Param::TauField) {
        Tensor t = base.detach().to(torch::kCPU, torch::kFloat64).contiguous();
        TORCH_CHECK(t.dim() == 2, "base tau field must be [ny][nx]");
        r.ny = (int)t.size(0);
        r.nx = (int)t.size(1);
        r.base_tau.assign(t.data_ptr<double>(), t.data_ptr<double>() + t.numel());
    } else {
        TORCH_CHECK(nx > 0 && ny > 0, "lattice size needed");
        r.nx = (int)nx;
        r.ny = (int)ny;
        Tensor w = base.detach().to(torch::kCPU, torch::kFloat32).contiguous();
        Tensor s = stats.detach().to(torch::kCPU, torch::kFloat32).contiguous();
        TORCH_CHECK(w.numel() == IPPI_MLP_PARAMS && s.numel() == IPPI_MLP_STATS, "network needs ",
                    IPPI_MLP_PARAMS, " weights and ", IPPI_MLP_STATS, " statistics");
        r.base_w.assign(w.data_ptr<float>(), w.data_ptr<float>() + w.numel());
        r.stats.assign(s.data_ptr<float>(), s.data_ptr<float>() + s.numel());
    }
    return hold;
}

struct RolloutFunction : public torch::autograd::Function<RolloutFunction> {
    static variable_list forward(AutogradContext* ctx, Tensor p, c10::intrusive_ptr<RolloutHolder> hold)
    {
        ctx->saved_data["rollout"] = hold;
        ctx->saved_data["dtype"] = static_cast<int64_t>(p.scalar_type());
        auto out = hold->r.run(p);
        return {out.first, out.second};
    }

    static variable_list backward(AutogradContext* ctx, variable_list g)
    {
        auto hold = ctx->saved_data["rollout"].toCustomClass<RolloutHolder>();
        const auto dtype = static_cast<c10::ScalarType>(ctx->saved_data["dtype"].toInt());
        Tensor grad = hold->r.grad(g[0], g[1]);
        if (hold->r.kind == Param::TauField) grad = grad.reshape({hold->r.ny, hold->r.nx});
        return {grad.to(dtype), Tensor()};
    }
};

}  // namespace ippi_torch

TORCH_LIBRARY(ippi_autograd, m) { m.class_<ippi_torch::RolloutHolder>("Rollout"); }

PYBIND11_MODULE(TORCH_EXTENSION_NAME, m)
{
    using namespace ippi_torch;
    m.doc() = "libtorch autograd Functions over the ippi_lbm adjoint (forward: checkpointed rollout; "
              "backward: the library's reverse sweep)";
    pybind11::class_<RolloutHolder, c10::intrusive_ptr<RolloutHolder>>(m, "Rollout")
        .def_property_readonly("nsteps", [](const RolloutHolder& x) { return x.r.nsteps; })
        .def_property_readonly("nbody", [](const RolloutHolder& x) { return x.r.nbody; })
        .def("__call__", [](c10::intrusive_ptr<RolloutHolder> self, const Tensor& p) {
            auto out = RolloutFunction::apply(p, self);
            return pybind11::make_tuple(out[0], out[1]);
        });
    m.def(
        "tau_field_rollout",
        [](int64_t handle, int64_t nsteps, int64_t t0, int64_t ckpt_every, const Tensor& base_tau) {
            return make_rollout(handle, Param::TauField, nsteps, t0, ckpt_every, base_tau, Tensor());
        },
        "Rollout differentiated with respect to the tau field [ny][nx] (IPPI_LES_FIELD); base_tau is "
        "the field in force on the lattice now; the starting state is the lattice's current state",
        pybind11::arg("handle"), pybind11::arg("nsteps"), pybind11::arg("t0"), pybind11::arg("ckpt_every"),
        pybind11::arg("base_tau"));
    m.def(
        "network_rollout",
        [](int64_t handle, int64_t nx, int64_t ny, int64_t nsteps, int64_t t0, int64_t ckpt_every,
           const Tensor& base_w, const Tensor& stats) {
            return make_rollout(handle, Param::Network, nsteps, t0, ckpt_every, base_w, stats, nx, ny);
        },
        "Rollout differentiated with respect to the learned network's FP32 weights [1313] "
        "(IPPI_LES_LEARNED) on an nx x ny lattice; base_w / stats are the network in force on the "
        "lattice now",
        pybind11::arg("handle"), pybind11::arg("nx"), pybind11::arg("ny"), pybind11::arg("nsteps"),
        pybind11::arg("t0"), pybind11::arg("ckpt_every"), pybind11::arg("base_w"), pybind11::arg("stats"));
}
