// Neuron-model plugins that put the reference engine's GPU time-driven models on
// this library.
//
// The reference loads neuron models by name through its model factory
// (src/neuron_model/NeuronModelFactory.cu:85-91,221-257); the time-driven GPU
// models derive from TimeDrivenNeuronModel_GPU_C_INTERFACE
// (include/neuron_model/TimeDrivenNeuronModel_GPU_C_INTERFACE.cuh:64-423).  The
// classes below keep the reference's LIF / AdEx / HH GPU interface classes for
// everything that describes a model -- .cfg parsing, parameter maps, integrator
// creation, PrintInfo -- and replace the state, the input and the update:
//
//   InitializeStates   the engine-side state arrays; at the first update, one
//                      population on a libedlut_b200 context (same model,
//                      integrator, BDF order, step and parameters) whose enabled
//                      conductance types are those the engine's synapses declared
//   ProcessInputSpike  each delivered weight queued with its target, type and
//                      arrival time (the engine then applies its STDP hook)
//   UpdateState        the step's queued arrivals folded into the conductances in
//                      delivery order on the device (eb_fold_arrivals), one
//                      integration step (eb_run), the spiking neurons flagged in
//                      the state's InternalSpike array the engine scans next
//   CheckSynapseType   AMPA / GABA / NMDA spike synapses; current synapses are
//                      outside this library's path
//
// so the engine's events, delivery, plasticity and outputs stay the reference's
// own and the neuron arithmetic is the library's (the reference CPU models', bit
// for bit).  The factory variant b200_factory.cu binds the reference's names
// LIFTimeDrivenModel_GPU, AdExTimeDrivenModel_GPU and HHTimeDrivenModel_GPU to
// these classes.
#include <cstdio>
#include <cstring>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>
#include <any>

#include <cuda_runtime.h>

#include "neuron_model/LIFTimeDrivenModel_GPU_C_INTERFACE.cuh"
#include "neuron_model/AdExTimeDrivenModel_GPU_C_INTERFACE.cuh"
#include "neuron_model/HHTimeDrivenModel_GPU_C_INTERFACE.cuh"
#include "neuron_model/VectorNeuronState_GPU_C_INTERFACE.cuh"
#include "neuron_model/CurrentSynapseModel.h"
#include "simulation/NetworkDescription.h"
#include "spike/Interconnection.h"
#include "openmp/openmp.h"

#include "edlut_b200.h"
#include "b200_models.h"

namespace {

void check(int rc, const char *what) {
    if (rc != EB_OK) throw std::runtime_error(std::string("libedlut_b200 ") + what + ": " + eb_last_error());
}

void check_cuda(cudaError_t e, const char *what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

// What distinguishes the three models here: the library's kind code, the .cfg
// parameter names in file order (the keys of the reference classes' parameter
// maps), and how many differential variables precede the conductances.
template <class Base> struct Traits;
template <> struct Traits<LIFTimeDrivenModel_GPU_C_INTERFACE> {
    static constexpr int kind = EB_LIF, nd = 1;
    static std::vector<const char *> keys() {
        return {"e_exc", "e_inh", "e_leak", "v_thr", "c_m", "tau_exc", "tau_inh", "tau_ref", "g_leak", "tau_nmda"};
    }
};
template <> struct Traits<AdExTimeDrivenModel_GPU_C_INTERFACE> {
    static constexpr int kind = EB_ADEX, nd = 2;
    static std::vector<const char *> keys() {
        return {"a", "b", "thr_slo_fac", "v_thr", "tau_w", "e_exc", "e_inh", "e_reset", "e_leak", "g_leak", "c_m",
                "tau_exc", "tau_inh", "tau_nmda"};
    }
};
template <> struct Traits<HHTimeDrivenModel_GPU_C_INTERFACE> {
    static constexpr int kind = EB_HH, nd = 4;
    static std::vector<const char *> keys() {
        return {"e_exc", "e_inh", "e_leak", "g_leak", "c_m", "v_thr", "tau_exc", "tau_inh", "tau_nmda", "g_na",
                "g_kd", "e_na", "e_k"};
    }
};

template <class Base>
class B200Model : public Base {
  public:
    B200Model() : Base() {}
    ~B200Model() override {
        if (ctx_) eb_ctx_destroy(ctx_);
        for (void *p : dev_) if (p) cudaFree(p);
    }

    static NeuronModel *CreateNeuronModel(ModelDescription desc) {
        B200Model *m = new B200Model();
        m->SetParameters(desc.param_map);
        return m;
    }

    // The engine initialises the states when it creates the layers, before it
    // reads the synapses that decide which conductance types are enabled
    // (src/spike/Network_GPU.cu:744-755): the library context is made at the first
    // update, when the types are known.
    void InitializeStates(int n, int queue) override {
        this->GPU_index = queue % NumberOfGPUs;
        device_ = GPUsIndex[this->GPU_index];
        check_cuda(cudaSetDevice(device_), "cudaSetDevice");
        check_cuda(cudaGetDeviceProperties(&this->prop, device_), "cudaGetDeviceProperties");
        n_ = n;
        // the engine-side state object: host arrays the engine reads (spike flags,
        // the monitored variables) mirroring the library's device state
        this->State_GPU = (VectorNeuronState_GPU_C_INTERFACE *)this->State;
        std::vector<float> init(this->State_GPU->GetNumberOfVariables(), 0.0f);
        this->State_GPU->InitializeStatesGPU(n, init.data(), this->N_TimeDependentNeuronState, this->prop);
        this->InitializeCurrentSynapsis(n);
    }

    InternalSpike *ProcessInputSpike(Interconnection *inter, double time) override {
        tgt_.push_back(inter->GetTargetNeuronModelIndex());
        type_.push_back((int8_t)inter->GetType());
        w_.push_back(inter->GetWeight());
        t_.push_back(time);
        return 0;
    }

    void ProcessInputCurrent(Interconnection *, Neuron *, float) override {
        throw std::runtime_error("current synapses are outside libedlut_b200's path");
    }

    bool UpdateState(int, double) override {
        check_cuda(cudaSetDevice(device_), "cudaSetDevice");
        if (!ctx_) make_context();
        const int64_t m = (int64_t)tgt_.size();
        if (m) {
            reserve(m);
            check_cuda(cudaMemcpyAsync(dev_[0], tgt_.data(), sizeof(int32_t) * m, cudaMemcpyHostToDevice, stream_), "copy");
            check_cuda(cudaMemcpyAsync(dev_[1], type_.data(), sizeof(int8_t) * m, cudaMemcpyHostToDevice, stream_), "copy");
            check_cuda(cudaMemcpyAsync(dev_[2], w_.data(), sizeof(float) * m, cudaMemcpyHostToDevice, stream_), "copy");
            check_cuda(cudaMemcpyAsync(dev_[3], t_.data(), sizeof(double) * m, cudaMemcpyHostToDevice, stream_), "copy");
            check(eb_fold_arrivals(stream_, m, (const int32_t *)dev_[0], (const int8_t *)dev_[1], (const float *)dev_[2],
                                   (const double *)dev_[3], n_, g_[0], g_[1], g_[2]),
                  "eb_fold_arrivals");
        }
        check(eb_run(ctx_, 1), "eb_run");  // synchronous: the host arrays above are free again
        tgt_.clear();
        type_.clear();
        w_.clear();
        t_.clear();
        int64_t ns = 0;
        int rc = eb_get_spikes(ctx_, 0, &ns, nullptr, nullptr);
        if (rc != EB_OK && rc != EB_ERR_OVERFLOW) check(rc, "eb_get_spikes");
        if (ns) {
            spk_step_.resize(ns);
            spk_cell_.resize(ns);
            check(eb_get_spikes(ctx_, ns, &ns, spk_step_.data(), spk_cell_.data()), "eb_get_spikes");
            bool *flag = this->State_GPU->getInternalSpike();
            for (int64_t s = 0; s < ns; ++s) flag[spk_cell_[s]] = true;
        }
        if (this->GetVectorNeuronState()->Get_Is_Monitored()) copy_state_to_host();
        return false;
    }

    bool CheckSynapseType(Interconnection *connection) override {
        const int type = connection->GetType();
        if (type == 0) this->EXC = true;
        else if (type == 1) this->INH = true;
        else if (type == 2) this->NMDA = true;
        else {
            std::fprintf(stderr, "%s: synapse type %d (current input) is outside libedlut_b200's path\n",
                         Base::GetName().c_str(), type);
            return false;
        }
        return true;
    }

    // The reference classes build device-side model objects here; the state lives
    // in the library context instead.
    void InitializeClassGPU2(int) override {}
    void InitializeVectorNeuronState_GPU2() override {}
    void DeleteClassGPU2() override {}

  private:
    // One population on a library context with this model's parameters in .cfg
    // order, integrator, BDF order and step, and the conductance types the
    // engine's synapses enabled (CheckSynapseType).
    void make_context() {
        std::map<std::string, boost::any> pm = this->GetParameters();
        std::vector<float> params;
        for (const char *k : Traits<Base>::keys()) params.push_back(boost::any_cast<float>(pm.at(k)));
        std::map<std::string, boost::any> im = this->integration_method_GPU->GetParameters();
        const std::string name = boost::any_cast<std::string>(im.at("name"));
        int integ = -1, order = 1;
        if (name == "Euler") integ = EB_EULER;
        else if (name == "RK2") integ = EB_RK2;
        else if (name == "RK4") integ = EB_RK4;
        else if (name == "BDF") { integ = EB_BDF; order = boost::any_cast<int>(im.at("bdf_order")); }
        else throw std::runtime_error("integration method " + name + " is outside libedlut_b200's path");
        const float dt = this->integration_method_GPU->GetIntegrationTimeStep();
        check(eb_ctx_create(device_, nullptr, &ctx_), "eb_ctx_create");
        check(eb_add_population(ctx_, Traits<Base>::kind, n_, integ, order, dt, params.data(), (int)params.size(), nullptr),
              "eb_add_population");
        const int mask = (this->EXC ? 1 : 0) | (this->INH ? 2 : 0) | (this->NMDA ? 4 : 0);
        check(eb_enable_conductances(ctx_, 0, mask), "eb_enable_conductances");
        check(eb_set_record_capacity(ctx_, 4 * (int64_t)n_ + 1024), "eb_set_record_capacity");
        check(eb_set_graph_steps(ctx_, 1), "eb_set_graph_steps");  // one step per UpdateState
        check(eb_finalize(ctx_, nullptr), "eb_finalize");
        void *st = nullptr;
        check(eb_stream(ctx_, &st), "eb_stream");
        stream_ = (cudaStream_t)st;
        for (int c = 0; c < 3; ++c)
            check(eb_population_state(ctx_, 0, Traits<Base>::nd + c, &g_[c]), "eb_population_state");
    }

    void reserve(int64_t m) {
        if (m <= cap_) return;
        const int64_t c = std::max<int64_t>(2 * m, 4096);
        const size_t sz[4] = {sizeof(int32_t), sizeof(int8_t), sizeof(float), sizeof(double)};
        for (int q = 0; q < 4; ++q) {
            if (dev_[q]) check_cuda(cudaFree(dev_[q]), "cudaFree");
            dev_[q] = nullptr;
            check_cuda(cudaMalloc(&dev_[q], sz[q] * (size_t)c), "cudaMalloc");
        }
        cap_ = c;
    }

    // VectorNeuronState_GPU_C_INTERFACE keeps variable v of neuron i at
    // VectorNeuronStates[v * n + i]; the library's state variables come in the
    // same model order (the current variable EXT_I, unsupported here, stays 0).
    void copy_state_to_host() {
        const int nv = this->State_GPU->GetNumberOfVariables();
        for (int v = 0; v < nv; ++v) {
            float *dst = this->State_GPU->VectorNeuronStates + (size_t)v * n_;
            if (eb_get_state(ctx_, 0, n_, v, dst) != EB_OK) std::memset(dst, 0, sizeof(float) * n_);
        }
    }

    eb_ctx *ctx_ = nullptr;
    cudaStream_t stream_ = nullptr;
    int device_ = 0, n_ = 0;
    float *g_[3] = {nullptr, nullptr, nullptr};
    void *dev_[4] = {nullptr, nullptr, nullptr, nullptr};
    int64_t cap_ = 0;
    std::vector<int32_t> tgt_;
    std::vector<int8_t> type_;
    std::vector<float> w_;
    std::vector<double> t_;
    std::vector<int64_t> spk_step_, spk_cell_;
};

}  // namespace

NeuronModel *b200_create_lif(ModelDescription d) { return B200Model<LIFTimeDrivenModel_GPU_C_INTERFACE>::CreateNeuronModel(d); }
NeuronModel *b200_create_adex(ModelDescription d) { return B200Model<AdExTimeDrivenModel_GPU_C_INTERFACE>::CreateNeuronModel(d); }
NeuronModel *b200_create_hh(ModelDescription d) { return B200Model<HHTimeDrivenModel_GPU_C_INTERFACE>::CreateNeuronModel(d); }
