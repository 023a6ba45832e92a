// Host runtime of the device-resident network: construction of the device
// tables, the K-step run loop (CUDA graphs), I/O, and the C ABI of
// include/edlut_b200.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "edlut_b200.h"
#include "eb_kernels.h"
#include "eb_record.h"
#include "eb_runtime.h"
#include "eb_tables.h"

using namespace eb;

static thread_local std::string g_err;

void eb::set_error(const char *fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
}

#define CK(call)                                                                              \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess) {                                                              \
            set_error("%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
            return EB_ERR_CUDA;                                                               \
        }                                                                                     \
    } while (0)

namespace {

int model_nv(int kind) { return kind == KIND_LIF ? 4 : kind == KIND_ADEX ? 5 : kind == KIND_HH ? 7 : 0; }
int model_nd(int kind) { return kind == KIND_LIF ? 1 : kind == KIND_ADEX ? 2 : kind == KIND_HH ? 4 : 0; }
int model_nparams(int kind) {
    return kind == KIND_LIF ? 10 : kind == KIND_ADEX ? 14 : kind == KIND_HH ? 13 : kind == KIND_POISSON ? 1 : 0;
}

}  // namespace

// ------------------------------------------------------------- allocation --
int eb_ctx::dalloc(void **p, size_t bytes) {
    if (bytes == 0) bytes = 16;
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) {
        set_error("cudaMalloc(%zu bytes) failed: %s", bytes, cudaGetErrorString(e));
        return EB_ERR_NOMEM;
    }
    allocs.push_back(*p);
    dev_bytes += (int64_t)bytes;
    return EB_OK;
}

void eb_ctx::dfree(void *p) {
    for (size_t i = 0; i < allocs.size(); ++i)
        if (allocs[i] == p) {
            allocs.erase(allocs.begin() + (long)i);
            cudaFree(p);
            return;
        }
}

void eb_ctx::dfree_all() {
    for (void *p : allocs) cudaFree(p);
    allocs.clear();
    dev_bytes = 0;
}

template <class T>
static int upload(eb_ctx *c, T **dptr, const std::vector<T> &h) {
    int rc = c->dalloc((void **)dptr, h.size() * sizeof(T));
    if (rc) return rc;
    if (!h.empty()) CK(cudaMemcpyAsync(*dptr, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, c->stream));
    return EB_OK;
}

// ----------------------------------------------------------- construction --
int eb_ctx::add_population(int kind, int64_t n, int integ, int bdf_order, float dt, const float *params,
                           int n_params, int64_t *out_first) {
    if (finalized) { set_error("eb_add_population after eb_finalize"); return EB_ERR_STATE; }
    if (n <= 0 || kind < KIND_INPUT || kind > KIND_POISSON) { set_error("bad population kind/size"); return EB_ERR_ARG; }
    HostPop p;
    p.kind = kind;
    p.n = n;
    p.first = n_neurons;
    if (kind == KIND_POISSON) {
        // PoissonGeneratorDeviceVector: one frequency, sampled every 0.1 ms
        // (sampling_period 0.1f / time scale 1000, PoissonGeneratorDeviceVector.cpp:26,137)
        if (n_params != 1 || !params) { set_error("a Poisson generator takes 1 parameter (frequency, Hz)"); return EB_ERR_ARG; }
        p.params.assign(params, params + 1);
        p.rates.assign(n, params[0]);
        p.dt = 0.1f / 1000.0f;
    } else if (kind != KIND_INPUT) {
        if (integ < INTEG_EULER || integ > INTEG_BDF) { set_error("unsupported integrator %d", integ); return EB_ERR_UNSUPPORTED; }
        if (integ == INTEG_BDF && (bdf_order < 1 || bdf_order > 6)) { set_error("BDF order must be 1..6"); return EB_ERR_ARG; }
        if (!(dt > 0.0f)) { set_error("integration step must be > 0"); return EB_ERR_ARG; }
        if (n_params != model_nparams(kind) || !params) {
            set_error("model kind %d takes %d parameters, got %d", kind, model_nparams(kind), n_params);
            return EB_ERR_ARG;
        }
        if (kind == KIND_LIF && params[7] >= 1.0e5f) { set_error("tau_ref must be < 1e5 ms"); return EB_ERR_UNSUPPORTED; }
        p.params.assign(params, params + n_params);
        p.integ = integ;
        p.bdf_order = integ == INTEG_BDF ? bdf_order : 0;
        p.dt = dt;
    }
    if (out_first) *out_first = p.first;
    n_neurons += n;
    pops.push_back(p);
    return EB_OK;
}

// Initial states of the Poisson generators' random generators, in the order the
// reference constructs them: RandomGenerator::srand(seed) (src/EDLUTKernel.cpp:88),
// one generator for the weights file (src/spike/Network.cpp:662), then one per
// generator neuron in Network::InitializeStates (src/spike/Network.cpp:274-283):
// model types in order of first appearance (layers with equal parameters share a
// type, Network.cpp:1023-1036), neurons of a type in index order; each takes the
// global seed, which then advances (include/simulation/RandomGenerator.h:61-68).
int eb_ctx::seed_generators() {
    uint32_t g = rng_seed & 0x7fffffffu;
    auto next = [](uint32_t v) { return (v * 765426813u + 54321u) & 0x7fffffffu; };
    g = next(g);  // the weights loader's generator
    std::vector<int> type_first;  // first population of each generator type
    std::vector<std::vector<size_t>> members;
    for (size_t q = 0; q < pops.size(); ++q) {
        if (pops[q].kind != KIND_POISSON) continue;
        size_t t = 0;
        while (t < type_first.size() && pops[type_first[t]].params != pops[q].params) ++t;
        if (t == type_first.size()) { type_first.push_back((int)q); members.emplace_back(); }
        members[t].push_back(q);
    }
    for (auto &mem : members)
        for (size_t q : mem) {
            std::vector<uint32_t> st(pops[q].n);
            for (auto &v : st) { v = g; g = next(g); }
            CK(cudaMemcpyAsync(pops[q].dev.lcg, st.data(), sizeof(uint32_t) * st.size(), cudaMemcpyHostToDevice, stream));
            CK(cudaStreamSynchronize(stream));
        }
    return EB_OK;
}

int eb_ctx::finalize(int64_t *out_sorted_perm) {
    if (finalized) { set_error("eb_finalize called twice"); return EB_ERR_STATE; }
    if (n_neurons <= 0) { set_error("no populations"); return EB_ERR_STATE; }
    const int64_t m = (int64_t)src.size();
    // step size shared by all model populations
    dt_f = 0.0f;
    has_generators = false;
    for (auto &p : pops) {
        if (p.kind == KIND_POISSON) has_generators = true;
        if (p.kind != KIND_INPUT && p.kind != KIND_POISSON) {
            if (dt_f == 0.0f) dt_f = p.dt;
            else if (p.dt != dt_f) { set_error("all model populations must share one integration step"); return EB_ERR_UNSUPPORTED; }
        }
    }
    if (dt_f == 0.0f) dt_f = has_generators ? 0.1f / 1000.0f : 1e-4f;
    if (has_generators && std::fabs((double)dt_f - (double)(0.1f / 1000.0f)) > 1e-9) {
        set_error("Poisson generators sample every 0.1 ms; the network's step is %g s", (double)dt_f);
        return EB_ERR_UNSUPPORTED;
    }
    dt_s = (double)dt_f;
    pop_of.assign(n_neurons, 0);
    for (size_t q = 0; q < pops.size(); ++q)
        for (int64_t i = 0; i < pops[q].n; ++i) pop_of[pops[q].first + i] = (int)q;
    // validate synapses, enable conductance types per target population
    std::vector<int64_t> units(m);
    int64_t max_units = 1;
    for (int64_t k = 0; k < m; ++k) {
        if (src[k] < 0 || src[k] >= n_neurons || tgt[k] < 0 || tgt[k] >= n_neurons) {
            set_error("synapse %lld: neuron index out of range", (long long)k);
            return EB_ERR_ARG;
        }
        HostPop &tp = pops[pop_of[tgt[k]]];
        if (tp.kind == KIND_INPUT || tp.kind == KIND_POISSON) {
            set_error("synapse %lld targets an input neuron", (long long)k);
            return EB_ERR_UNSUPPORTED;
        }
        if (stype[k] < 0 || stype[k] > 2) {
            set_error("synapse %lld: type %d (only 0 AMPA, 1 GABA, 2 NMDA spike synapses)", (long long)k, stype[k]);
            return EB_ERR_UNSUPPORTED;
        }
        if (rule[k] >= (int32_t)rules.size()) { set_error("synapse %lld: learning rule %d undefined", (long long)k, rule[k]); return EB_ERR_ARG; }
        tp.en |= 1 << stype[k];
        units[k] = delay_units(delay[k]);
        if (units[k] > 65535) { set_error("delay above 6.5535 s"); return EB_ERR_UNSUPPORTED; }
        max_units = std::max(max_units, units[k]);
    }
    // reference synapse order: (source, delay, target), ties by original index
    std::vector<int64_t> ord(m);
    std::iota(ord.begin(), ord.end(), 0);
    std::stable_sort(ord.begin(), ord.end(), [&](int64_t a, int64_t b) {
        if (src[a] != src[b]) return src[a] < src[b];
        if (units[a] != units[b]) return units[a] < units[b];
        return tgt[a] < tgt[b];
    });
    if (out_sorted_perm) std::copy(ord.begin(), ord.end(), out_sorted_perm);
    spos_of.assign(m, 0);
    for (int64_t s = 0; s < m; ++s) spos_of[ord[s]] = s;
    std::vector<int64_t> out_ptr(n_neurons + 1, 0);
    for (int64_t k = 0; k < m; ++k) out_ptr[src[k] + 1]++;
    for (int64_t i = 0; i < n_neurons; ++i) out_ptr[i + 1] += out_ptr[i];
    // target-major order: per target, plastic first, then reference order
    std::vector<int64_t> in_ptr(n_neurons + 1, 0), plastic_end(n_neurons, 0);
    std::vector<int64_t> indeg_in(n_neurons, 0);
    for (int64_t k = 0; k < m; ++k) {
        in_ptr[tgt[k] + 1]++;
        if (pops[pop_of[src[k]]].kind == KIND_INPUT) indeg_in[tgt[k]]++;
    }
    for (int64_t i = 0; i < n_neurons; ++i) in_ptr[i + 1] += in_ptr[i];
    std::vector<int64_t> tord(ord);  // already by spos; stable partition by (target, plastic first)
    std::stable_sort(tord.begin(), tord.end(), [&](int64_t a, int64_t b) {
        if (tgt[a] != tgt[b]) return tgt[a] < tgt[b];
        return (rule[a] >= 0) > (rule[b] >= 0);
    });
    tpos_of.assign(m, 0);
    for (int64_t t = 0; t < m; ++t) tpos_of[tord[t]] = t;
    for (int64_t i = 0; i < n_neurons; ++i) {
        int64_t e = in_ptr[i];
        while (e < in_ptr[i + 1] && rule[tord[e]] >= 0) ++e;
        plastic_end[i] = e;
    }
    // source-major device arrays
    std::vector<uint32_t> h_out_tgt(m), h_out_tpos(m);
    std::vector<uint16_t> h_out_units(m);
    for (int64_t s = 0; s < m; ++s) {
        int64_t k = ord[s];
        h_out_tgt[s] = (uint32_t)tgt[k];
        h_out_tpos[s] = (uint32_t)tpos_of[k];
        h_out_units[s] = (uint16_t)units[k];
    }
    std::vector<int64_t> grp_ptr(n_neurons + 1, 0);
    std::vector<uint16_t> grp_units;
    for (int64_t i = 0; i < n_neurons; ++i) {
        grp_ptr[i] = (int64_t)grp_units.size();
        for (int64_t s = out_ptr[i]; s < out_ptr[i + 1]; ++s)
            if (s == out_ptr[i] || h_out_units[s] != h_out_units[s - 1]) grp_units.push_back(h_out_units[s]);
    }
    grp_ptr[n_neurons] = (int64_t)grp_units.size();
    // target-major device arrays
    std::vector<float> h_w(m), h_maxw(m);
    std::vector<uint8_t> h_type(m);
    std::vector<int8_t> h_rule(m);
    for (int64_t t = 0; t < m; ++t) {
        int64_t k = tord[t];
        h_w[t] = weight[k];
        h_maxw[t] = max_weight[k];
        h_type[t] = (uint8_t)stype[k];
        h_rule[t] = (int8_t)rule[k];
    }
    // bucket capacities
    std::vector<uint32_t> h_cap(n_neurons);
    std::vector<int64_t> h_cap_base(n_neurons);
    int64_t cap_total = 0;
    for (int64_t i = 0; i < n_neurons; ++i) {
        int64_t indeg = in_ptr[i + 1] - in_ptr[i];
        int64_t c = (indeg - indeg_in[i]) + (int64_t)input_multiplicity * indeg_in[i];
        c = std::min<int64_t>(c, (int64_t)bucket_limit);
        h_cap[i] = (uint32_t)c;
        h_cap_base[i] = cap_total;
        cap_total += c;
    }
    // delay ring: arrival at most ceil(max delay / dt) + 1 steps ahead, plus
    // kMaxFuse slots so that a launch can run that many steps of a population
    // (see plan_chains); a power of two, so the kernels take the slot of step k as
    // k & (R - 1)
    const double dmax = (double)max_units * 0.0001;
    const int r_min = (int)std::ceil(dmax / dt_s) + 3 + kMaxFuse;
    R = 1;
    while (R < r_min) R <<= 1;

    int rc;
    cudaStream_t st = stream;
    NetDev N;
    memset(&N, 0, sizeof(N));
    N.n_neurons = n_neurons;
    N.R = R;
    if ((rc = dalloc((void **)&d_step, sizeof(int64_t)))) return rc;
    CK(cudaMemsetAsync(d_step, 0, sizeof(int64_t), st));
    N.step = d_step;
    if ((rc = dalloc((void **)&N.cnt, sizeof(uint32_t) * (size_t)R * n_neurons))) return rc;
    CK(cudaMemsetAsync(N.cnt, 0, sizeof(uint32_t) * (size_t)R * n_neurons, st));
    if ((rc = dalloc((void **)&N.rec, sizeof(Arrival) * (size_t)R * std::max<int64_t>(cap_total, 1)))) return rc;
    N.cap_total = cap_total;
    if ((rc = upload(this, (int64_t **)&N.cap_base, h_cap_base))) return rc;
    if ((rc = upload(this, (uint32_t **)&N.cap, h_cap))) return rc;
    if ((rc = upload(this, (int64_t **)&N.out_ptr, out_ptr))) return rc;
    if ((rc = upload(this, (uint32_t **)&N.out_tgt, h_out_tgt))) return rc;
    if ((rc = upload(this, (uint32_t **)&N.out_tpos, h_out_tpos))) return rc;
    if ((rc = upload(this, (uint16_t **)&N.out_units, h_out_units))) return rc;
    if ((rc = upload(this, (int64_t **)&N.grp_ptr, grp_ptr))) return rc;
    if ((rc = upload(this, (uint16_t **)&N.grp_units, grp_units))) return rc;
    if ((rc = upload(this, (int64_t **)&N.in_ptr, in_ptr))) return rc;
    if ((rc = upload(this, (int64_t **)&N.plastic_end, plastic_end))) return rc;
    {
        std::vector<SynRec> hs(m);
        for (int64_t k = 0; k < m; ++k) {
            SynRec &r = hs[k];
            memset(&r, 0, sizeof(r));
            r.w = h_w[k];
            r.maxw = h_maxw[k];
            r.stype = h_type[k];
            r.rule = h_rule[k];
        }
        if ((rc = upload(this, &N.syn, hs))) return rc;
    }
    std::vector<float> rp;
    for (auto &r : rules) {
        rp.push_back(r[0]); rp.push_back(r[1]); rp.push_back(r[2]); rp.push_back(r[3]);
        rp.push_back(1.0f / r[1]);  // inv_LTPTau = 1.0f/tau (STDPState.cpp:23-26)
        rp.push_back(1.0f / r[3]);
    }
    if (rp.empty()) rp.assign(6, 0.0f);
    if ((rc = upload(this, (float **)&N.rule_par, rp))) return rc;
    if ((rc = upload(this, (float **)&N.exp_table, make_exp_table()))) return rc;
    N.expt_aux = exp_table_aux();
    if ((rc = dalloc((void **)&N.flags, sizeof(uint32_t)))) return rc;
    CK(cudaMemsetAsync(N.flags, 0, sizeof(uint32_t), st));
    if ((rc = dalloc((void **)&N.events, sizeof(unsigned long long) * pops.size()))) return rc;
    CK(cudaMemsetAsync(N.events, 0, sizeof(unsigned long long) * pops.size(), st));
    if ((rc = dalloc((void **)&N.rec_count, sizeof(unsigned long long)))) return rc;
    CK(cudaMemsetAsync(N.rec_count, 0, sizeof(unsigned long long), st));
    N.rec_cap = rec_cap;
    if (rec_cap > 0 && (rc = dalloc((void **)&N.rec_buf, sizeof(unsigned long long) * (size_t)rec_cap))) return rc;
    has_inputs = false;
    for (auto &p : pops)
        if (p.kind == KIND_INPUT) has_inputs = true;
    // input fan-out may run beside the neuron updates when no input delivery can
    // reach the step being updated: every input synapse delay exceeds the step
    {
        int64_t min_units = INT64_MAX, max_out_in = 0;
        for (int64_t i = 0; i < n_neurons; ++i) {
            if (pops[pop_of[i]].kind != KIND_INPUT) continue;
            max_out_in = std::max(max_out_in, out_ptr[i + 1] - out_ptr[i]);
            for (int64_t s = out_ptr[i]; s < out_ptr[i + 1]; ++s) min_units = std::min<int64_t>(min_units, h_out_units[s]);
        }
        inputs_concurrent = min_units == INT64_MAX || (double)min_units * 0.0001 > dt_s;
        input_threads = (int)std::min<int64_t>(256, std::max<int64_t>(32, (max_out_in + 31) / 32 * 32));
    }
    net = N;

    // populations
    for (auto &p : pops) {
        if (p.kind == KIND_INPUT) continue;
        PopDev &D = p.dev;
        memset(&D, 0, sizeof(D));
        D.kind = p.kind;
        D.integ = p.integ;
        D.bdf_order = p.bdf_order;
        D.ndiff = model_nd(p.kind);
        D.nvars = model_nv(p.kind);
        D.en = p.en;
        D.events = N.events + (&p - pops.data());
        D.first = p.first;
        D.n = p.n;
        for (size_t j = 0; j < p.params.size(); ++j) D.p[j] = p.params[j];
        D.dt_s = p.dt;
        D.dt_ms = p.dt * 1000.0f;  // IntegrationMethodFast.h:192
        if (p.kind == KIND_POISSON) {
            // threshold (double)frequency * step, step = (double)(0.1f / 1000): the
            // comparison PoissonGeneratorDeviceVector.cpp:61 makes with frand()
            std::vector<double> thr(p.n);
            for (int64_t i = 0; i < p.n; ++i) thr[i] = (double)p.rates[i] * (double)p.dt;
            if ((rc = upload(this, (double **)&D.pthr, thr))) return rc;
            if ((rc = dalloc((void **)&D.lcg, sizeof(uint32_t) * (size_t)p.n))) return rc;
        } else {
            const float *pr = p.params.data();
            float tau[3] = {0, 0, 0};
            float init[kMaxVars] = {0};
            std::vector<float> nmda;
            if (p.kind == KIND_LIF) {
                D.inv_c_m = inv_double(pr[4]);
                tau[0] = pr[5]; tau[1] = pr[6]; tau[2] = pr[9];
                init[0] = pr[2];
                nmda = make_nmda_table(pr[0], pr[1], &D.nmda_aux);
            } else if (p.kind == KIND_ADEX) {
                D.inv_c_m = inv_double(pr[10]);
                D.inv_slope = inv_double(pr[2]);
                D.inv_tau_w = inv_double(pr[4]);
                D.adex_vmax = pr[3] + 6 * pr[2];
                D.adex_glslope = pr[9] * pr[2];
                tau[0] = pr[11]; tau[1] = pr[12]; tau[2] = pr[13];
                init[0] = pr[8];
                nmda = make_nmda_table(pr[5], pr[6], &D.nmda_aux);
            } else {
                D.inv_c_m = inv_double(pr[4]);
                tau[0] = pr[6]; tau[1] = pr[7]; tau[2] = pr[8];
                std::vector<float> hh = make_hh_table(pr[5]);
                D.hh_aux = hh_table_aux();
                // HHTimeDrivenModel::InitializeStates (HHTimeDrivenModel.cpp:141-166)
                int pos = (int)((pr[2] - (-90.0f)) * D.hh_aux);
                if (pos < 0) pos = 0; else if (pos > kHHTable - 1) pos = kHHTable - 1;
                const float *v = hh.data() + (size_t)pos * 6;
                init[0] = pr[2];
                init[1] = v[0] / (v[0] + v[1]);
                init[2] = v[2] / (v[2] + v[3]);
                init[3] = v[4] / (v[4] + v[5]);
                if ((rc = upload(this, (float **)&D.hh_table, hh))) return rc;
                nmda = make_nmda_table(pr[0], pr[1], &D.nmda_aux);
            }
            if ((rc = upload(this, (float **)&D.nmda_table, nmda))) return rc;
            const float el = (p.integ == INTEG_RK4) ? D.dt_ms * 0.5f : D.dt_ms;  // RK4.h:362
            for (int c = 0; c < 3; ++c) D.decay[c] = decay_factor(el, tau[c]);
            bdf_coefficients(D.bdf_coef);
            memcpy(D.init, init, sizeof(init));
            D.expt_aux = exp_table_aux();
            D.exp_table = N.exp_table;
            const int nd = D.ndiff;
            for (int v = 0; v < D.nvars; ++v) {
                bool stored = v < nd || (p.en & (1 << (v - nd)));
                if (!stored) { D.x[v] = nullptr; continue; }
                std::vector<float> h(p.n, init[v]);
                if ((rc = upload(this, &D.x[v], h))) return rc;
            }
            if (p.kind == KIND_LIF) {
                std::vector<int32_t> h(p.n, -1);
                if ((rc = upload(this, &D.refr, h))) return rc;
            }
            if (p.integ == INTEG_BDF) {
                std::vector<int8_t> hs(p.n, 0);
                if ((rc = upload(this, &D.bdf_state, hs))) return rc;
                std::vector<float> hd((size_t)p.bdf_order * nd * p.n, 0.0f);
                if ((rc = upload(this, &D.bdf_D, hd))) return rc;
                std::vector<float> hp((size_t)std::max(p.bdf_order - 1, 1) * nd * p.n, 0.0f);
                if ((rc = upload(this, &D.bdf_P, hp))) return rc;
            }
        }
        if ((rc = dalloc((void **)&D.spk, sizeof(uint32_t) * (size_t)p.n))) return rc;
        if ((rc = dalloc((void **)&D.spk_count, 2 * sizeof(uint32_t)))) return rc;
        CK(cudaMemsetAsync(D.spk_count, 0, 2 * sizeof(uint32_t), st));
        uint32_t maxcap = 0;
        int64_t max_plastic = 0, max_indeg = 0;
        for (int64_t i = p.first; i < p.first + p.n; ++i) {
            maxcap = std::max(maxcap, h_cap[i]);
            max_plastic = std::max(max_plastic, plastic_end[i] - in_ptr[i]);
            max_indeg = std::max(max_indeg, in_ptr[i + 1] - in_ptr[i]);
        }
        // a block per neuron pays off when a step brings many arrivals (in-degree x
        // rate x dt); the bucket capacity is only the worst case of one step
        D.wide = maxcap > 16 && max_indeg > wide_indegree ? 1 : 0;
        p.has_plastic_in = max_plastic > 0;
        p.post_chunks = (int)((max_plastic + kPostThreads - 1) / kPostThreads);
        if (p.has_plastic_in) {
            // deferred post-synaptic STDP (graph path): a ring of recent spike times
            lazy_post = true;
            if ((rc = dalloc((void **)&D.post_t, sizeof(double) * (size_t)kPostRing * p.n))) return rc;
            if ((rc = dalloc((void **)&D.post_n, sizeof(uint32_t) * (size_t)p.n))) return rc;
            if ((rc = dalloc((void **)&D.post_flushed, sizeof(uint32_t) * (size_t)p.n))) return rc;
            CK(cudaMemsetAsync(D.post_t, 0, sizeof(double) * (size_t)kPostRing * p.n, st));
            CK(cudaMemsetAsync(D.post_n, 0, sizeof(uint32_t) * (size_t)p.n, st));
            CK(cudaMemsetAsync(D.post_flushed, 0, sizeof(uint32_t) * (size_t)p.n, st));
            if ((rc = dalloc((void **)&D.flush_list, sizeof(uint32_t) * (size_t)(p.n + 1)))) return rc;
            CK(cudaMemsetAsync(D.flush_list, 0, sizeof(uint32_t) * (size_t)(p.n + 1), st));
            // one rule on every plastic input: decay factors of the spike intervals
            int rule_one = -2;
            for (int64_t i = p.first; i < p.first + p.n && rule_one != -1; ++i)
                for (int64_t e = in_ptr[i]; e < plastic_end[i]; ++e) {
                    const int r = rule[tord[e]];
                    if (rule_one == -2) rule_one = r;
                    else if (rule_one != r) { rule_one = -1; break; }
                }
            D.post_rule = rule_one >= 0 ? rule_one : -1;
            if (D.post_rule >= 0) {
                if ((rc = dalloc((void **)&D.post_f, sizeof(DecayPair) * (size_t)kPostRing * p.n))) return rc;
                CK(cudaMemsetAsync(D.post_f, 0, sizeof(DecayPair) * (size_t)kPostRing * p.n, st));
            }
        } else {
            D.post_rule = -1;
        }
        p.has_out = false;
        int64_t max_out = 0, in_from_inputs = 0;
        for (int64_t i = p.first; i < p.first + p.n; ++i) {
            if (out_ptr[i + 1] > out_ptr[i]) p.has_out = true;
            max_out = std::max(max_out, out_ptr[i + 1] - out_ptr[i]);
            in_from_inputs += indeg_in[i];
        }
        p.push_threads = (int)std::min<int64_t>(256, std::max<int64_t>(32, (max_out + 31) / 32 * 32));
        D.may_repeat = in_from_inputs > 0 ? 1 : 0;
    }
    plan_chains(out_ptr, h_out_tgt, h_out_units);
    if ((rc = seed_generators())) return rc;
    // dynamic state copied by eb_snapshot / eb_restore
    dyn.clear();
    dyn.push_back({d_step, sizeof(int64_t)});
    dyn.push_back({net.cnt, sizeof(uint32_t) * (size_t)R * n_neurons});
    dyn.push_back({net.rec, sizeof(Arrival) * (size_t)R * std::max<int64_t>(net.cap_total, 1)});
    dyn.push_back({net.syn, sizeof(SynRec) * (size_t)std::max<int64_t>(m, 1)});
    dyn.push_back({net.events, sizeof(unsigned long long) * pops.size()});
    for (auto &p : pops) {
        if (p.kind == KIND_INPUT) continue;
        for (int v = 0; v < p.dev.nvars; ++v)
            if (p.dev.x[v]) dyn.push_back({p.dev.x[v], sizeof(float) * (size_t)p.n});
        if (p.dev.refr) dyn.push_back({p.dev.refr, sizeof(int32_t) * (size_t)p.n});
        if (p.dev.bdf_state) {
            const int nd = p.dev.ndiff;
            dyn.push_back({p.dev.bdf_state, sizeof(int8_t) * (size_t)p.n});
            dyn.push_back({p.dev.bdf_D, sizeof(float) * (size_t)p.bdf_order * nd * p.n});
            dyn.push_back({p.dev.bdf_P, sizeof(float) * (size_t)std::max(p.bdf_order - 1, 1) * nd * p.n});
        }
        dyn.push_back({p.dev.spk_count, 2 * sizeof(uint32_t)});
        if (p.dev.lcg) dyn.push_back({p.dev.lcg, sizeof(uint32_t) * (size_t)p.n});
        if (p.dev.post_t) {
            dyn.push_back({p.dev.post_t, sizeof(double) * (size_t)kPostRing * p.n});
            dyn.push_back({p.dev.post_n, sizeof(uint32_t) * (size_t)p.n});
            dyn.push_back({p.dev.post_flushed, sizeof(uint32_t) * (size_t)p.n});
            if (p.dev.post_f) dyn.push_back({p.dev.post_f, sizeof(DecayPair) * (size_t)kPostRing * p.n});
        }
    }
    for (int q = 0; q < std::max(4, (int)chain_pop.size() - 1); ++q) {
        cudaStream_t ss;
        CK(cudaStreamCreateWithFlags(&ss, cudaStreamNonBlocking));
        side.push_back(ss);
    }
    for (int q = 0; q < std::max(8, (int)chain_pop.size()); ++q) {
        cudaEvent_t a, b;
        CK(cudaEventCreateWithFlags(&a, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&b, cudaEventDisableTiming));
        fork_ev.push_back(a);
        join_ev.push_back(b);
    }
    if ((rc = setup_persistent())) return rc;
    CK(prepare_update_kernels());
    CK(cudaStreamSynchronize(st));
    finalized = true;
    steps_done = 0;
    // time grid and input bookkeeping
    t_host.assign(1, 0.0);
    in_start_host.assign(2, 0);
    return EB_OK;
}

// --------------------------------------------------------------- run loop --
// Grow the device step-time table and input-range table to cover step kmax.
int eb_ctx::ensure_tables(int64_t kmax) {
    while ((int64_t)t_host.size() <= kmax) {
        double t = t_host.back() + (double)dt_f;  // TimeEventUpdateNeurons.cpp:115
        t_host.push_back(t);
    }
    if (has_generators) {
        // generators keep their own grid, t'_k = t'_{k-1} + (double)(0.1f / 1000); their
        // k-th draw belongs to step k while t_k <= t'_k < t_{k+1}
        const double gstep = (double)(0.1f / 1000.0f);
        while ((int64_t)tgen_host.size() <= kmax) {
            const int64_t k = (int64_t)tgen_host.size();
            const double t = tgen_host.back() + gstep;
            if (k + 1 < (int64_t)t_host.size() && !(t_host[k] <= t && t < t_host[k + 1])) {
                set_error("Poisson generator step %lld falls outside the network step (grids drifted apart)", (long long)k);
                return EB_ERR_UNSUPPORTED;
            }
            tgen_host.push_back(t);
        }
    }
    int64_t need = kmax + 1;
    if (need > tcap) {
        int64_t ncap = std::max<int64_t>(need * 2, 4096);
        double *nt = nullptr;
        int64_t *ni = nullptr;
        int rc;
        if ((rc = dalloc((void **)&nt, sizeof(double) * (size_t)ncap))) return rc;
        if ((rc = dalloc((void **)&ni, sizeof(int64_t) * (size_t)(ncap + 1)))) return rc;
        if (has_generators && (rc = dalloc((void **)&d_tgen, sizeof(double) * (size_t)ncap))) return rc;
        CK(cudaMemsetAsync(ni, 0, sizeof(int64_t) * (size_t)(ncap + 1), stream));
        if (d_instart && tcap > 0)
            CK(cudaMemcpyAsync(ni, d_instart, sizeof(int64_t) * (size_t)(tcap + 1), cudaMemcpyDeviceToDevice, stream));
        d_tstep = nt;
        d_instart = ni;
        tcap = ncap;
        tstep_uploaded = 0;
        graphs_valid = false;
    }
    if (tstep_uploaded < need) {
        CK(cudaMemcpyAsync(d_tstep + tstep_uploaded, t_host.data() + tstep_uploaded,
                           sizeof(double) * (size_t)(need - tstep_uploaded), cudaMemcpyHostToDevice, stream));
        if (has_generators)
            CK(cudaMemcpyAsync(d_tgen + tstep_uploaded, tgen_host.data() + tstep_uploaded,
                               sizeof(double) * (size_t)(need - tstep_uploaded), cudaMemcpyHostToDevice, stream));
        tstep_uploaded = need;
    }
    net.tstep = d_tstep;
    net.tgen = d_tgen;
    net.in_start = d_instart;
    return EB_OK;
}

// Move pending input spikes with time < t_{k_end} to the device and fill the
// input ranges of steps k0+1 .. k_end+1.
int eb_ctx::stage_inputs(int64_t k0, int64_t k_end) {
    if (k_end <= staged_until && pending.empty()) return EB_OK;
    const double tend = t_host[k_end];
    std::vector<double> nt;
    std::vector<uint32_t> nc;
    std::vector<PendingIn> rest;
    for (auto &p : pending) {
        if ((double)p.t < tend) { nt.push_back((double)p.t); nc.push_back((uint32_t)p.cell); }
        else rest.push_back(p);
    }
    pending.swap(rest);
    // After eb_restore, new inputs can precede inputs staged for the abandoned
    // timeline: merge them into the staged list in time order and re-stage it.
    if (!nt.empty() && !in_times_host.empty() && nt.front() < in_times_host.back()) {
        std::vector<double> mt;
        std::vector<uint32_t> mc;
        mt.reserve(in_times_host.size() + nt.size());
        mc.reserve(in_times_host.size() + nt.size());
        size_t a = 0, b = 0;
        while (a < in_times_host.size() || b < nt.size()) {
            if (b == nt.size() || (a < in_times_host.size() && in_times_host[a] <= nt[b])) {
                mt.push_back(in_times_host[a]);
                mc.push_back(in_cells_host[a++]);
            } else {
                mt.push_back(nt[b]);
                mc.push_back(nc[b++]);
            }
        }
        in_times_host.clear();
        in_cells_host.clear();
        in_total = 0;
        nt.swap(mt);
        nc.swap(mc);
        staged_until = k_end;  // input ranges of later steps are recomputed when they are staged
    }
    if (!nt.empty()) {
        int64_t need = in_total + (int64_t)nt.size();
        if (need > in_cap) {
            int64_t ncap = std::max<int64_t>(need * 2, 1 << 16);
            double *dt = nullptr;
            uint32_t *dc = nullptr;
            int rc;
            if ((rc = dalloc((void **)&dt, sizeof(double) * (size_t)ncap))) return rc;
            if ((rc = dalloc((void **)&dc, sizeof(uint32_t) * (size_t)ncap))) return rc;
            if (in_total) {
                CK(cudaMemcpyAsync(dt, d_in_time, sizeof(double) * (size_t)in_total, cudaMemcpyDeviceToDevice, stream));
                CK(cudaMemcpyAsync(dc, d_in_cell, sizeof(uint32_t) * (size_t)in_total, cudaMemcpyDeviceToDevice, stream));
            }
            d_in_time = dt;
            d_in_cell = dc;
            in_cap = ncap;
            graphs_valid = false;
        }
        CK(cudaMemcpyAsync(d_in_time + in_total, nt.data(), sizeof(double) * nt.size(), cudaMemcpyHostToDevice, stream));
        CK(cudaMemcpyAsync(d_in_cell + in_total, nc.data(), sizeof(uint32_t) * nc.size(), cudaMemcpyHostToDevice, stream));
        in_times_host.insert(in_times_host.end(), nt.begin(), nt.end());
        in_cells_host.insert(in_cells_host.end(), nc.begin(), nc.end());
        in_total += (int64_t)nt.size();
    }
    // in_start[k] = first staged input with time >= t_{k-1}
    std::vector<int64_t> h(k_end - k0 + 1);
    for (int64_t k = k0 + 1; k <= k_end + 1; ++k) {
        double lo = t_host[k - 1];
        h[k - k0 - 1] = std::lower_bound(in_times_host.begin(), in_times_host.end(), lo) - in_times_host.begin();
    }
    CK(cudaMemcpyAsync(d_instart + k0 + 1, h.data(), sizeof(int64_t) * h.size(), cudaMemcpyHostToDevice, stream));
    net.in_time = d_in_time;
    net.in_cell = d_in_cell;
    staged_until = std::max(staged_until, k_end);
    return EB_OK;
}

// Profiling: the steps are captured into a graph whose kernels are bracketed
// by event-record nodes on the stream (branch) each kernel runs on, so the GPU
// timestamps every launch without the host in the loop.
void eb_ctx::prof_begin(int kind, int pop, cudaEvent_t *a) {
    (void)kind; (void)pop;
    if (!profile) return;
    if (ev_pool.empty()) {
        cudaEvent_t e;
        cudaEventCreate(&e);
        ev_pool.push_back(e);
    }
    *a = ev_pool.back();
    ev_pool.pop_back();
    cudaEventRecordWithFlags(*a, prof_stream, cudaEventRecordExternal);
}

void eb_ctx::prof_end(int kind, int pop, cudaEvent_t a) {
    if (!profile) return;
    if (ev_pool.empty()) {
        cudaEvent_t e;
        cudaEventCreate(&e);
        ev_pool.push_back(e);
    }
    cudaEvent_t b = ev_pool.back();
    ev_pool.pop_back();
    cudaEventRecordWithFlags(b, prof_stream, cudaEventRecordExternal);
    prof_pending.push_back({kind, pop, a, b});
}

int eb_ctx::prof_collect() {
    for (auto &r : prof_pending) {
        float ms = 0.0f;
        CK(cudaEventElapsedTime(&ms, r.a, r.b));
        bool found = false;
        for (auto &s : prof_sum)
            if (s.kind == r.kind && s.pop == r.pop) { s.launches++; s.ms += ms; found = true; }
        if (!found) prof_sum.push_back({r.kind, r.pop, 1, (double)ms});
        ev_pool.push_back(r.a);
        ev_pool.push_back(r.b);
    }
    prof_pending.clear();
    return EB_OK;
}

// Run the launches of one phase on parallel branches (main stream + side
// streams, joined back into the main stream); sequential when profiling.
void eb_ctx::fork_join(std::vector<std::function<void(cudaStream_t)>> &work) {
    if (work.empty()) return;
    if (work.size() == 1) {
        for (auto &f : work) f(stream);
        return;
    }
    const size_t nb = std::min(work.size(), side.size() + 1);
    cudaEventRecord(fork_ev[0], stream);
    for (size_t b = 1; b < nb; ++b) cudaStreamWaitEvent(side[b - 1], fork_ev[0], 0);
    for (size_t i = 0; i < work.size(); ++i) {
        const size_t b = i % nb;
        work[i](b == 0 ? stream : side[b - 1]);
    }
    for (size_t b = 1; b < nb; ++b) {
        cudaEventRecord(join_ev[b], side[b - 1]);
        cudaStreamWaitEvent(stream, join_ev[b], 0);
    }
}

// Deferred post-synaptic STDP: apply the noted spikes to the synapses (on the
// context stream, profiled as kind 4).  A partial flush (at least every kPostGraph
// steps) only takes the neurons whose rings could overflow before the next one; a
// full flush (before the host reads or writes weights, or the eager-STDP
// persistent kernel runs) takes every neuron with a pending spike.
void eb_ctx::enqueue_flush(bool full) {
    steps_since_flush = 0;
    for (size_t q = 0; q < pops.size(); ++q) enqueue_flush_pop((int)q, full, stream);
}

void eb_ctx::enqueue_flush_pop(int q, bool full, cudaStream_t s) {
    const auto &p = pops[q];
    if (!p.dev.post_t) return;
    const uint32_t keep = full ? 0u : (uint32_t)(kPostRing - kPostGraph);
    cudaEvent_t a = nullptr;
    prof_stream = s;
    prof_begin(4, q, &a);
    enq_count += 3;
    launch_flush_post(p.dev, net, std::max(1, p.post_chunks), keep, 148 * 8, s);
    prof_end(4, q, a);
}

int eb_ctx::flush_post() {
    if (!lazy_post || !finalized) return EB_OK;
    enqueue_flush(true);
    CK(cudaGetLastError());
    return EB_OK;
}

// Captured graph of K steps (cached per K; see build_graph).
eb_ctx::CachedGraph *eb_ctx::graph_for(int K) {
    if (!graphs_valid) {
        for (auto &g : graph_cache) cudaGraphExecDestroy(g.exec);
        graph_cache.clear();
        graphs_valid = true;
    }
    for (auto &g : graph_cache)
        if (g.K == K) return &g;
    if (graph_cache.size() >= 8) {
        cudaGraphExecDestroy(graph_cache.front().exec);
        graph_cache.erase(graph_cache.begin());
    }
    if (build_graph(K)) return nullptr;
    return &graph_cache.back();
}

void eb_ctx::enqueue_step(int rel) {
    const int fan_blocks = 148 * 4;
    const double inv_dt = 1.0 / dt_s;
    std::vector<std::function<void(cudaStream_t)>> phase;
    auto timed = [this](int kind, int pop, std::function<void(cudaStream_t)> f) {
        return [this, kind, pop, f](cudaStream_t s) {
            cudaEvent_t a = nullptr;
            prof_stream = s;
            prof_begin(kind, pop, &a);
            enq_count++;
            f(s);
            prof_end(kind, pop, a);
        };
    };
    if (has_inputs) {
        auto f = timed(0, -1, [this, rel, inv_dt, fan_blocks](cudaStream_t s) {
            launch_input_push(net, rel, 1, inv_dt, fan_blocks, input_threads, s);
        });
        if (inputs_concurrent) phase.push_back(f);
        else f(stream);
    }
    for (size_t q = 0; q < pops.size(); ++q) {
        if (pops[q].kind == KIND_INPUT) continue;
        // spikes fan out inside the update kernel (arrivals land at step k+1 or later)
        const double push_inv_dt = pops[q].has_out ? inv_dt : 0.0;
        phase.push_back(timed(1, (int)q, [this, q, rel, push_inv_dt](cudaStream_t s) {
            launch_update(pops[q].dev, net, rel, 1, push_inv_dt, s);
        }));
    }
    fork_join(phase);
    phase.clear();
    for (size_t q = 0; q < pops.size(); ++q) {
        auto &p = pops[q];
        if (p.kind == KIND_INPUT) continue;
        if (p.has_plastic_in && !p.dev.post_t)
            phase.push_back(timed(2, (int)q, [this, q, rel, fan_blocks](cudaStream_t s) {
                launch_post_stdp(pops[q].dev, net, rel, pops[q].post_chunks, fan_blocks, s);
            }));

    }
    fork_join(phase);
}

// Decide whether the persistent kernel can run this network and prepare its
// arguments: at most kMaxPersistPops model populations, cooperative launch
// support, and at least one resident block per SM.
int eb_ctx::setup_persistent() {
    persist_ok = false;
    int coop = 0, nsm = 0;
    CK(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device));
    CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device));
    int n_model = 0;
    persist_class = 0;
    memset(&pinfo, 0, sizeof(pinfo));
    pinfo.spin_limit = barrier_spin_limit;
    pinfo.withhold = barrier_withhold ? 1 : 0;
    for (auto &p : pops) {
        if (p.kind == KIND_INPUT) continue;
        if (p.kind == KIND_POISSON) return EB_OK;  // generators run on the graph path only
        if (n_model < kMaxPersistPops) {
            if (p.has_out) pinfo.has_out |= 1u << n_model;
            if (p.has_plastic_in) pinfo.has_plastic |= 1u << n_model;
            pinfo.post_chunks[n_model] = std::max(1, p.post_chunks);
        }
        persist_class = std::max(persist_class, persist_class_of(p.kind, p.integ));
        n_model++;
    }
    if (!coop || n_model == 0 || n_model > kMaxPersistPops) return EB_OK;
    const int bps = persistent_blocks_per_sm(persist_class);
    if (bps < 1) return EB_OK;
    persist_grid = bps * nsm;
    pinfo.n_pops = n_model;
    {
        int j = 0, q = 0;
        std::vector<int> wide, narrow;
        for (auto &p : pops) {
            if (p.kind == KIND_INPUT) continue;
            (p.dev.wide ? wide : narrow).push_back(q++);
        }
        for (int w : wide) pinfo.order[j++] = w;
        for (int w : narrow) pinfo.order[j++] = w;
        pinfo.n_wide = (int)wide.size();
    }
    pinfo.has_inputs = has_inputs ? 1 : 0;
    pinfo.inputs_concurrent = inputs_concurrent ? 1 : 0;
    pinfo.inv_dt = 1.0 / dt_s;
    int rc;
    bar_words = (size_t)((persist_grid + 15) / 16 + 2) * 32;  // generation, root, one line per group
    if ((rc = dalloc((void **)&pinfo.bar, bar_words * sizeof(unsigned)))) return rc;
    CK(cudaMemsetAsync(pinfo.bar, 0, bar_words * sizeof(unsigned), stream));
    if ((rc = dalloc((void **)&d_pops, sizeof(PopDev) * (size_t)n_model))) return rc;
    if ((rc = dalloc((void **)&pinfo.queue, 4 * 16 * sizeof(unsigned long long)))) return rc;
    CK(cudaMemsetAsync(pinfo.queue, 0, 4 * 16 * sizeof(unsigned long long), stream));
    pops_dirty = true;
    persist_ok = true;
    return EB_OK;
}

// Chains of the captured graph: one per model population, one for all input
// neurons (chain 0, so that its launch of step r is captured before the updates of
// step r).  Population B's update at step k reads and clears bucket slot k; a
// source chain A writes, at step j, arrivals for steps j + lo .. j + hi, lo and hi
// bounding the arrival offsets of the delays from A to B with a step of margin for
// rounding of the time grid.  So B(k) waits for A(k - lo) -- every arrival of step
// k is in place -- and A(j) waits for B(j - (R - hi)) -- the slot it fills for
// step j + hi has been cleared for its previous use, R steps before.  Everything
// else a chain touches belongs to its own population (state, spike lists, the
// target-major synapse records and the deferred post-synaptic rings), so the
// chains need no other edge and the steps run exactly as in step order.
//
// A launch may run S consecutive steps of a chain (its neurons' state stays in
// registers) when no step inside the window needs another step of the same
// window: every lag into a model population (lo) and every slot-reuse lag (R -
// hi), its own population's included, is at least S.  Input chains may feed a
// window of the same index (lo < S): they are captured first and wait for nothing
// of that window.
void eb_ctx::plan_chains(const std::vector<int64_t> &out_ptr, const std::vector<uint32_t> &out_tgt,
                         const std::vector<uint16_t> &out_units) {
    chain_pop.clear();
    chain_deps.clear();
    std::vector<int> chain_of(pops.size(), -1);
    if (has_inputs) chain_pop.push_back(-1);
    for (size_t q = 0; q < pops.size(); ++q) {
        if (pops[q].kind == KIND_INPUT) chain_of[q] = 0;
        else { chain_of[q] = (int)chain_pop.size(); chain_pop.push_back((int)q); }
    }
    const int nc = (int)chain_pop.size();
    std::vector<int64_t> umin((size_t)nc * nc, INT64_MAX), umax((size_t)nc * nc, -1);
    for (int64_t i = 0; i < n_neurons; ++i) {
        const int a = chain_of[pop_of[i]];
        for (int64_t s = out_ptr[i]; s < out_ptr[i + 1]; ++s) {
            const int b = chain_of[pop_of[out_tgt[s]]];
            const size_t e = (size_t)a * nc + b;
            umin[e] = std::min<int64_t>(umin[e], out_units[s]);
            umax[e] = std::max<int64_t>(umax[e], out_units[s]);
        }
    }
    chain_deps.assign(nc, {});
    int fuse = kMaxFuse;
    for (int a = 0; a < nc; ++a)
        for (int b = 0; b < nc; ++b) {
            const size_t e = (size_t)a * nc + b;
            if (umax[e] < 0) continue;
            const bool from_inputs = chain_pop[a] < 0;
            // inputs of step j are the spikes of [t_{j-1}, t_j): one step earlier than a
            // neuron's spike at t_j, so one step less of lower bound
            const int lo = std::max(from_inputs ? 0 : 1,
                                    (int)std::floor((double)umin[e] * 0.0001 / dt_s) - (from_inputs ? 2 : 1));
            const int hi = (int)std::ceil((double)umax[e] * 0.0001 / dt_s) + 2;
            if (!from_inputs) fuse = std::min(fuse, lo);
            fuse = std::min(fuse, R - hi);
            if (a == b) continue;
            chain_deps[b].push_back({a, lo});
            chain_deps[a].push_back({b, R - hi});
        }
    chain_fuse = 1;
    while (chain_fuse * 2 <= fuse) chain_fuse *= 2;
    chains_ok = nc >= 2 && nc <= 8;
    for (auto &p : pops)
        if (p.kind != KIND_INPUT && p.has_plastic_in && !p.dev.post_t) chains_ok = false;  // eager post phase
    for (auto &d : chain_deps)
        for (auto &x : d)
            if (x.lag < 0 || (x.lag == 0 && chain_pop[x.other] >= 0)) chains_ok = false;
}

// K steps as per-population chains (see plan_chains), joined at the end; each
// launch runs a window of S steps (S divides K).  A population's partial flush of
// deferred post-synaptic STDP only touches its own synapses and rings, so it runs
// in the population's chain every kPostGraph steps (and at the end of the graph).
void eb_ctx::enqueue_chains(int K) {
    const int nc = (int)chain_pop.size();
    int S = chain_fuse;
    while (K % S) S >>= 1;
    const int W = K / S;
    while ((int)chain_ev.size() < nc * W) {
        cudaEvent_t e;
        cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
        chain_ev.push_back(e);
    }
    auto ev = [&](int c, int w) { return chain_ev[(size_t)c * W + w]; };
    auto strm = [&](int c) { return c == 0 ? stream : side[c - 1]; };
    const double inv_dt = 1.0 / dt_s;
    cudaEventRecord(fork_ev[0], stream);
    for (int c = 1; c < nc; ++c) cudaStreamWaitEvent(strm(c), fork_ev[0], 0);
    for (int w = 0; w < W; ++w)
        for (int c = 0; c < nc; ++c) {
            cudaStream_t s = strm(c);
            for (auto &d : chain_deps[c]) {
                // the window's last step needs step x of the other chain
                const int x = w * S + S - 1 - d.lag;
                if (x >= 0) cudaStreamWaitEvent(s, ev(d.other, x / S), 0);
            }
            const int q = chain_pop[c];
            cudaEvent_t a = nullptr;
            prof_stream = s;
            prof_begin(q < 0 ? 0 : 1, q, &a);
            if (q < 0) {
                launch_input_push(net, w * S, S, inv_dt, 148 * 4, input_threads, s);
            } else {
                const double push_inv_dt = pops[q].has_out ? inv_dt : 0.0;
                launch_update(pops[q].dev, net, w * S, S, push_inv_dt, s);
            }
            prof_end(q < 0 ? 0 : 1, q, a);
            enq_count++;
            const int end = (w + 1) * S;
            if (q >= 0 && lazy_post && (end % kPostGraph == 0 || end == K)) enqueue_flush_pop(q, false, s);
            cudaEventRecord(ev(c, w), s);
        }
    for (int c = 1; c < nc; ++c) {
        cudaEventRecord(join_ev[c], strm(c));
        cudaStreamWaitEvent(stream, join_ev[c], 0);
    }
}

int eb_ctx::build_graph(int K) {
    const int since_flush = steps_since_flush;  // capturing flushes nothing yet
    cudaGraph_t g;
    CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
    enq_count = 0;
    if (chains_ok && chains_enabled) {
        enqueue_chains(K);
    } else {
        for (int r = 0; r < K; ++r) {
            enqueue_step(r);
            if (lazy_post && ((r + 1) % kPostGraph == 0 || r + 1 == K)) enqueue_flush(false);
        }
    }
    const int kernels = enq_count + 1;
    launch_advance(d_step, K, stream);
    CK(cudaStreamEndCapture(stream, &g));
    cudaGraphExec_t exec = nullptr;
    cudaError_t e = cudaGraphInstantiate(&exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) { set_error("cudaGraphInstantiate: %s", cudaGetErrorString(e)); return EB_ERR_CUDA; }
    graph_cache.push_back({K, kernels, exec});
    steps_since_flush = since_flush;
    return EB_OK;
}

int eb_ctx::run_async(int64_t n) {
    if (!finalized) { set_error("eb_run before eb_finalize"); return EB_ERR_STATE; }
    if (n <= 0) return EB_OK;
    const int64_t k0 = steps_done, k_end = k0 + n;
    int rc;
    if ((rc = ensure_tables(k_end + R + 8))) return rc;
    if ((rc = stage_inputs(k0, k_end))) return rc;
    if (trace_pending) {
        net.trace_k0 = k0 + 1;
        trace_pending = false;
        graphs_valid = false;
    }
    const int K = graph_steps > 0 ? graph_steps : kDefaultGraph;
    int64_t done = 0;
    if (persistent && persist_ok && !profile) {
        if (lazy_post) enqueue_flush(true);  // the persistent kernel applies post-synaptic STDP eagerly
        if (pops_dirty) {
            // the persistent kernel applies post-synaptic STDP at each spike (its own
            // phase); the flush above left no deferred spike pending
            std::vector<PopDev> h;
            for (auto &p : pops)
                if (p.kind != KIND_INPUT) {
                    h.push_back(p.dev);
                    h.back().post_t = nullptr;
                    h.back().post_n = nullptr;
                    h.back().post_flushed = nullptr;
                    h.back().post_f = nullptr;
                }
            CK(cudaMemcpyAsync(d_pops, h.data(), sizeof(PopDev) * h.size(), cudaMemcpyHostToDevice, stream));
            pops_dirty = false;
        }
        const int64_t chunk = 1000;
        while (done < n) {
            const int k = (int)std::min<int64_t>(chunk, n - done);
            cudaError_t e = launch_persistent(persist_class, d_pops, pinfo, net, k, persist_grid, stream);
            if (e != cudaSuccess) { set_error("persistent kernel launch: %s", cudaGetErrorString(e)); return EB_ERR_CUDA; }
            launches += 1;
            done += k;
        }
        steps_done = k_end;
        return EB_OK;
    }
    if (profile) {
        // one graph of all n steps with timestamped kernels (events are reused only
        // after prof_collect, so n bounds the number of events in flight)
        cudaGraph_t g;
        cudaGraphExec_t ge;
        CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        enq_count = 0;
        if (lazy_post && steps_since_flush) enqueue_flush(false);
        if (chains_ok && chains_enabled && n <= (1 << 20)) {
            enqueue_chains((int)n);  // the graph path's launches, each bracketed by events
        } else {
            for (int64_t r = 0; r < n; ++r) {
                enqueue_step((int)r);
                if (lazy_post && (r + 1) % kPostGraph == 0) enqueue_flush(false);
            }
            if (lazy_post) enqueue_flush(false);
        }
        launch_advance(d_step, (int)n, stream);
        CK(cudaStreamEndCapture(stream, &g));
        CK(cudaGraphInstantiate(&ge, g, 0));
        cudaGraphDestroy(g);
        CK(cudaGraphLaunch(ge, stream));
        CK(cudaStreamSynchronize(stream));
        cudaGraphExecDestroy(ge);
        launches += enq_count + 1;
        steps_done = k_end;
        return EB_OK;
    }
    // whole graphs of K steps, then one graph of the remainder when it is long
    // enough to pay for its capture (cached, so repeated run lengths reuse it)
    for (int pass = 0; pass < 2 && K > 1; ++pass) {
        const int Kp = pass == 0 ? K : (int)(n - done);
        if (n - done < Kp || Kp < kMinGraph) continue;
        CachedGraph *g = graph_for(Kp);
        if (!g) return EB_ERR_CUDA;
        if (lazy_post && steps_since_flush) {  // a graph starts with every ring at most kPostRing - kPostGraph full
            enq_count = 0;
            enqueue_flush(false);
            launches += enq_count;
        }
        while (n - done >= Kp) {
            CK(cudaGraphLaunch(g->exec, stream));
            launches += g->kernels;
            done += Kp;
        }
        steps_since_flush = 0;  // every graph ends with a partial flush
    }
    while (done < n) {
        enq_count = 0;
        enqueue_step(0);
        launch_advance(d_step, 1, stream);
        if (lazy_post && ++steps_since_flush == kPostGraph) enqueue_flush(false);
        launches += enq_count + 1;
        done++;
    }
    CK(cudaGetLastError());
    steps_done = k_end;
    return EB_OK;
}

int eb_ctx::sync() {
    CK(cudaStreamSynchronize(stream));
    if (profile) {
        int rc = prof_collect();
        if (rc) return rc;
    }
    uint32_t f = 0;
    CK(cudaMemcpy(&f, net.flags, sizeof(f), cudaMemcpyDeviceToHost));
    if (f) {
        CK(cudaMemset(net.flags, 0, sizeof(uint32_t)));
        if (f & FLAG_BDF_SINGULAR) { set_error("BDF Newton matrix not invertible"); return EB_ERR_NUMERIC; }
        if (f & FLAG_BUCKET_OVERFLOW) {
            set_error("arrival bucket overflow: a neuron received more spikes in one step than its bucket holds "
                      "(raise eb_set_bucket_limit)");
            return EB_ERR_OVERFLOW;
        }
        if (f & FLAG_RECORD_OVERFLOW) { set_error("spike recording buffer full (drain with eb_get_spikes or raise eb_set_record_capacity)"); return EB_ERR_OVERFLOW; }
        if (f & FLAG_SPIKELIST_OVERFLOW) { set_error("internal spike list overflow"); return EB_ERR_OVERFLOW; }
        if (f & FLAG_BARRIER_TIMEOUT) {
            // blocks gave up part-way through a barrier: reset its counters and the
            // item queues, so the next launch starts from a clean barrier
            if (pinfo.bar) CK(cudaMemset(pinfo.bar, 0, bar_words * sizeof(unsigned)));
            if (pinfo.queue) CK(cudaMemset(pinfo.queue, 0, 4 * 16 * sizeof(unsigned long long)));
            set_error("persistent kernel: grid barrier wait timed out (the run stopped part-way; restore a "
                      "snapshot before continuing)");
            return EB_ERR_CUDA;
        }
        if (f & FLAG_PERSIST_UNSUPPORTED) { set_error("persistent kernel: integrator outside its compiled class"); return EB_ERR_STATE; }
        if (f & FLAG_MONITOR_OVERFLOW) {
            set_error("state monitor: more deliveries into monitored neurons in one chunk than its log holds "
                      "(raise the delivery capacity of eb_open_monitor)");
            return EB_ERR_OVERFLOW;
        }
    }
    return EB_OK;
}

int eb_set_barrier_wait(eb_ctx *ctx, uint64_t spin_limit, int withhold_first_block) {
    if (!ctx || spin_limit == 0) { set_error("bad argument"); return EB_ERR_ARG; }
    ctx->barrier_spin_limit = spin_limit;
    ctx->barrier_withhold = withhold_first_block != 0;
    ctx->pinfo.spin_limit = spin_limit;
    ctx->pinfo.withhold = withhold_first_block != 0 ? 1 : 0;
    return EB_OK;
}

int eb_ctx::snapshot(int slot) {
    if (!finalized) { set_error("not finalized"); return EB_ERR_STATE; }
    std::vector<void *> *bufs = nullptr;
    for (auto &s : snapshots)
        if (s.first == slot) bufs = &s.second;
    if (!bufs) {
        snapshots.push_back({slot, {}});
        bufs = &snapshots.back().second;
        for (auto &d : dyn) {
            void *p = nullptr;
            int rc = dalloc(&p, d.second);
            if (rc) return rc;
            bufs->push_back(p);
        }
    }
    for (size_t i = 0; i < dyn.size(); ++i)
        CK(cudaMemcpyAsync((*bufs)[i], dyn[i].first, dyn[i].second, cudaMemcpyDeviceToDevice, stream));
    bool found = false;
    for (auto &h : snap_host)
        if (h.slot == slot) {
            h.steps_done = steps_done;
            h.spikes_drained = spikes_drained;
            h.steps_since_flush = steps_since_flush;
            found = true;
        }
    if (!found) snap_host.push_back({slot, steps_done, spikes_drained, steps_since_flush});
    CK(cudaStreamSynchronize(stream));
    return EB_OK;
}

int eb_ctx::restore(int slot) {
    std::vector<void *> *bufs = nullptr;
    for (auto &s : snapshots)
        if (s.first == slot) bufs = &s.second;
    if (!bufs) { set_error("no snapshot in slot %d", slot); return EB_ERR_STATE; }
    for (size_t i = 0; i < dyn.size(); ++i)
        CK(cudaMemcpyAsync(dyn[i].first, (*bufs)[i], dyn[i].second, cudaMemcpyDeviceToDevice, stream));
    for (auto &h : snap_host)
        if (h.slot == slot) {
            steps_done = h.steps_done;
            spikes_drained = h.spikes_drained;
            steps_since_flush = h.steps_since_flush;
        }
    CK(cudaMemsetAsync(net.rec_count, 0, sizeof(unsigned long long), stream));
    rec_step_lo = steps_done;
    CK(cudaStreamSynchronize(stream));
    return EB_OK;
}

eb_ctx::~eb_ctx() {
    for (auto &g : graph_cache) cudaGraphExecDestroy(g.exec);
    for (auto s : side) cudaStreamDestroy(s);
    for (auto e : chain_ev) cudaEventDestroy(e);
    for (auto e : fork_ev) cudaEventDestroy(e);
    for (auto e : join_ev) cudaEventDestroy(e);
    for (auto &r : prof_pending) { ev_pool.push_back(r.a); ev_pool.push_back(r.b); }
    for (auto e : ev_pool) cudaEventDestroy(e);
    if (mon_file) std::fclose(mon_file);
    dfree_all();
    if (rec_host) cudaFreeHost(rec_host);
    if (own_stream && stream) cudaStreamDestroy(stream);
}

// ================================================================== C ABI ==
extern "C" {

const char *eb_last_error(void) { return g_err.c_str(); }
const char *eb_version(void) { return "edlut_b200 0.1 (sm_100a)"; }

int eb_ctx_create(int device, void *stream, eb_ctx **out) {
    if (!out) { set_error("null out"); return EB_ERR_ARG; }
    *out = nullptr;
    CK(cudaSetDevice(device));
    eb_ctx *c = new eb_ctx();
    c->device = device;
    if (stream) {
        c->stream = (cudaStream_t)stream;
        c->own_stream = false;
    } else {
        cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) { delete c; set_error("cudaStreamCreate: %s", cudaGetErrorString(e)); return EB_ERR_CUDA; }
        c->own_stream = true;
    }
    *out = c;
    return EB_OK;
}

int eb_ctx_destroy(eb_ctx *ctx) {
    if (!ctx) return EB_OK;
    cudaSetDevice(ctx->device);
    delete ctx;
    return EB_OK;
}

int eb_add_population(eb_ctx *ctx, int kind, int64_t n, int integrator, int bdf_order, float dt_s,
                      const float *params, int n_params, int64_t *out_first) {
    if (!ctx) { set_error("null context"); return EB_ERR_ARG; }
    return ctx->add_population(kind, n, integrator, bdf_order, dt_s, params, n_params, out_first);
}

int eb_add_stdp_rule(eb_ctx *ctx, float max_ltp, float tau_ltp, float max_ltd, float tau_ltd, int *out_rule) {
    if (!ctx) { set_error("null context"); return EB_ERR_ARG; }
    if (ctx->finalized) { set_error("eb_add_stdp_rule after eb_finalize"); return EB_ERR_STATE; }
    if (!(tau_ltp > 0) || !(tau_ltd > 0)) { set_error("STDP time constants must be > 0"); return EB_ERR_ARG; }
    ctx->rules.push_back({max_ltp, tau_ltp, max_ltd, tau_ltd});
    if (out_rule) *out_rule = (int)ctx->rules.size() - 1;
    return EB_OK;
}

int eb_set_connectivity(eb_ctx *ctx, int64_t m, const int64_t *src, const int64_t *tgt, const float *delay_s,
                        const int32_t *type, const float *weight, const float *max_weight, const int32_t *rule) {
    if (!ctx) { set_error("null context"); return EB_ERR_ARG; }
    if (ctx->finalized) { set_error("eb_set_connectivity after eb_finalize"); return EB_ERR_STATE; }
    if (m < 0 || (m > 0 && (!src || !tgt || !delay_s || !type || !weight || !max_weight))) {
        set_error("bad connectivity arrays");
        return EB_ERR_ARG;
    }
    if (m >= (int64_t)UINT32_MAX) { set_error("more than 2^32-1 synapses"); return EB_ERR_UNSUPPORTED; }
    ctx->src.assign(src, src + m);
    ctx->tgt.assign(tgt, tgt + m);
    ctx->delay.assign(delay_s, delay_s + m);
    ctx->stype.assign(type, type + m);
    ctx->weight.assign(weight, weight + m);
    ctx->max_weight.assign(max_weight, max_weight + m);
    if (rule) ctx->rule.assign(rule, rule + m);
    else ctx->rule.assign(m, -1);
    return EB_OK;
}

int eb_set_wide_indegree(eb_ctx *ctx, int64_t indegree) {
    if (!ctx || indegree < 0) { set_error("bad argument"); return EB_ERR_ARG; }
    if (ctx->finalized) { set_error("eb_set_wide_indegree after eb_finalize"); return EB_ERR_STATE; }
    ctx->wide_indegree = indegree;
    return EB_OK;
}

int eb_set_bucket_limit(eb_ctx *ctx, uint32_t max_per_target, uint32_t input_multiplicity) {
    if (!ctx) { set_error("null context"); return EB_ERR_ARG; }
    if (ctx->finalized) { set_error("eb_set_bucket_limit after eb_finalize"); return EB_ERR_STATE; }
    if (max_per_target) ctx->bucket_limit = max_per_target;
    if (input_multiplicity) ctx->input_multiplicity = input_multiplicity;
    return EB_OK;
}

int eb_finalize(eb_ctx *ctx, int64_t *out_sorted_perm) {
    if (!ctx) { set_error("null context"); return EB_ERR_ARG; }
    CK(cudaSetDevice(ctx->device));
    return ctx->finalize(out_sorted_perm);
}

int eb_inject_spikes(eb_ctx *ctx, int64_t n, const float *time_s, const int64_t *cell) {
    if (!ctx) { set_error("null context"); return EB_ERR_ARG; }
    if (n < 0 || (n > 0 && (!time_s || !cell))) { set_error("bad input arrays"); return EB_ERR_ARG; }
    double now = ctx->finalized && !ctx->t_host.empty() ? ctx->t_host[std::min<int64_t>(ctx->steps_done, (int64_t)ctx->t_host.size() - 1)] : 0.0;
    for (int64_t i = 0; i < n; ++i) {
        if (cell[i] < 0 || cell[i] >= ctx->n_neurons) { set_error("input spike %lld: neuron out of range", (long long)i); return EB_ERR_ARG; }
        if ((double)time_s[i] < now || !(time_s[i] >= 0.0f)) {
            set_error("input spike %lld at %g s precedes the simulation time %g s", (long long)i, (double)time_s[i], now);
            return EB_ERR_ARG;
        }
    }
    for (int64_t i = 0; i < n; ++i) {
        ctx->pending.push_back({time_s[i], cell[i], ctx->pending_seq++});
        // a model neuron used as an input source can deliver twice in one step
        if (ctx->finalized && ctx->pops[ctx->pop_of[cell[i]]].kind != KIND_INPUT) {
            for (auto &p : ctx->pops) p.dev.may_repeat = 1;
            ctx->graphs_valid = false;
            ctx->pops_dirty = true;
        }
    }
    std::stable_sort(ctx->pending.begin(), ctx->pending.end(), [](const PendingIn &a, const PendingIn &b) {
        if (a.t != b.t) return a.t < b.t;
        return a.seq < b.seq;
    });
    return EB_OK;
}

int eb_set_timeline(eb_ctx *ctx, int steps) {
    if (!ctx || steps < 0) { set_error("bad argument"); return EB_ERR_ARG; }
    if (!ctx->persist_ok) { set_error("persistent kernel not in use"); return EB_ERR_STATE; }
    if (steps > 0) {
        int rc = ctx->dalloc((void **)&ctx->pinfo.tl, sizeof(unsigned long long) * (size_t)steps * 6 * ctx->persist_grid);
        if (rc) return rc;
    } else {
        ctx->pinfo.tl = nullptr;
    }
    ctx->pinfo.tl_steps = steps;
    return EB_OK;
}

int eb_get_timeline(eb_ctx *ctx, int *grid, unsigned long long *out) {
    if (!ctx || !grid) { set_error("bad argument"); return EB_ERR_ARG; }
    *grid = ctx->persist_grid;
    if (out && ctx->pinfo.tl) {
        CK(cudaStreamSynchronize(ctx->stream));
        CK(cudaMemcpy(out, ctx->pinfo.tl, sizeof(unsigned long long) * (size_t)ctx->pinfo.tl_steps * 6 * ctx->persist_grid,
                      cudaMemcpyDeviceToHost));
    }
    return EB_OK;
}

int eb_set_persistent(eb_ctx *ctx, int on) {
    if (!ctx) { set_error("null context"); return EB_ERR_ARG; }
    ctx->persistent = on != 0;
    return EB_OK;
}

int eb_set_graph_steps(eb_ctx *ctx, int graph_steps) {
    if (!ctx || graph_steps < 0) { set_error("bad argument"); return EB_ERR_ARG; }
    ctx->graph_steps = graph_steps;
    return EB_OK;
}

int eb_run_async(eb_ctx *ctx, int64_t n_steps) {
    if (!ctx) { set_error("null context"); return EB_ERR_ARG; }
    if (ctx->mon_file) { set_error("eb_run_async while the state monitor is open (eb_run writes it)"); return EB_ERR_STATE; }
    CK(cudaSetDevice(ctx->device));
    return ctx->run_async(n_steps);
}

int eb_sync(eb_ctx *ctx) {
    if (!ctx) { set_error("null context"); return EB_ERR_ARG; }
    return ctx->sync();
}

int eb_run(eb_ctx *ctx, int64_t n_steps) {
    if (ctx && ctx->mon_file) {
        CK(cudaSetDevice(ctx->device));
        return ctx->run_monitored(n_steps);
    }
    int rc = eb_run_async(ctx, n_steps);
    if (rc) return rc;
    return ctx->sync();
}

int eb_set_record_capacity(eb_ctx *ctx, int64_t cap) {
    if (!ctx || cap < 0) { set_error("bad argument"); return EB_ERR_ARG; }
    if (ctx->finalized) { set_error("eb_set_record_capacity after eb_finalize"); return EB_ERR_STATE; }
    ctx->rec_cap = cap;
    return EB_OK;
}

int eb_get_spikes(eb_ctx *ctx, int64_t cap, int64_t *n, int64_t *step, int64_t *cell) {
    if (!ctx || !n) { set_error("bad argument"); return EB_ERR_ARG; }
    if (!ctx->finalized) { set_error("not finalized"); return EB_ERR_STATE; }
    CK(cudaStreamSynchronize(ctx->stream));
    unsigned long long cnt = 0;
    CK(cudaMemcpy(&cnt, ctx->net.rec_count, sizeof(cnt), cudaMemcpyDeviceToHost));
    int64_t have = (int64_t)std::min<unsigned long long>(cnt, (unsigned long long)ctx->rec_cap);
    *n = have;
    if (have > cap) { set_error("eb_get_spikes: %lld spikes, buffer holds %lld", (long long)have, (long long)cap); return EB_ERR_OVERFLOW; }
    if (have > ((int64_t)1 << 31)) { set_error("eb_get_spikes: more than 2^31 recorded spikes"); return EB_ERR_OVERFLOW; }
    // sort on the device (eb_record.cu), copy through a pinned buffer, unpack
    // while checking the order and the ranges
    const int64_t s_lo = ctx->rec_step_lo, s_hi = ctx->steps_done;
    if (have > 0) {
        int rc;
        if (have > ctx->rec_sort_cap) {
            const int64_t ncap = std::max<int64_t>(have + have / 2, 1 << 16);
            if (ctx->rec_tmp) { ctx->dfree(ctx->rec_tmp); ctx->rec_tmp = nullptr; }
            if (ctx->rec_hist) { ctx->dfree(ctx->rec_hist); ctx->rec_hist = nullptr; }
            if (ctx->rec_host) { cudaFreeHost(ctx->rec_host); ctx->rec_host = nullptr; }
            ctx->rec_sort_cap = 0;
            if ((rc = ctx->dalloc((void **)&ctx->rec_tmp, sizeof(unsigned long long) * (size_t)ncap))) return rc;
            if ((rc = ctx->dalloc((void **)&ctx->rec_hist, sizeof(uint32_t) * eb::record_sort_hist_words(ncap)))) return rc;
            CK(cudaHostAlloc((void **)&ctx->rec_host, sizeof(unsigned long long) * (size_t)ncap, cudaHostAllocDefault));
            ctx->rec_sort_cap = ncap;
        }
        unsigned long long *sorted = nullptr;
        CK(eb::sort_record(ctx->net.rec_buf, ctx->rec_tmp, ctx->rec_hist, have, s_lo, s_hi, ctx->n_neurons, ctx->stream,
                           &sorted));
        ctx->launches += eb::record_sort_launches(have, s_lo, s_hi, ctx->n_neurons);
        CK(cudaMemcpyAsync(ctx->rec_host, sorted, sizeof(unsigned long long) * (size_t)have, cudaMemcpyDeviceToHost,
                           ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
    }
    const unsigned long long *h = ctx->rec_host;
    for (int64_t i = 0; i < have; ++i) {
        const int64_t k = (int64_t)(h[i] >> 32), c = (int64_t)(h[i] & 0xffffffffull);
        if ((i > 0 && h[i] <= h[i - 1]) || k <= s_lo || k > s_hi || c >= ctx->n_neurons) {
            set_error("eb_get_spikes: spike record %lld (step %lld, neuron %lld) out of order or range", (long long)i,
                      (long long)k, (long long)c);
            return EB_ERR_STATE;
        }
        if (step) step[i] = k;
        if (cell) cell[i] = c;
    }
    ctx->spikes_drained += have;
    ctx->rec_step_lo = s_hi;
    CK(cudaMemset(ctx->net.rec_count, 0, sizeof(unsigned long long)));
    return EB_OK;
}

int eb_step_time(eb_ctx *ctx, int64_t k, double *t) {
    if (!ctx || !t || k < 0) { set_error("bad argument"); return EB_ERR_ARG; }
    while ((int64_t)ctx->t_host.size() <= k) ctx->t_host.push_back(ctx->t_host.back() + (double)ctx->dt_f);
    *t = ctx->t_host[k];
    return EB_OK;
}

static int state_io(eb_ctx *ctx, int64_t first, int64_t n, int var, float *buf, bool get) {
    if (!ctx || n < 0 || first < 0 || first + n > ctx->n_neurons || var < 0 || var >= kMaxVars) {
        set_error("bad state range");
        return EB_ERR_ARG;
    }
    if (!ctx->finalized) { set_error("not finalized"); return EB_ERR_STATE; }
    CK(cudaStreamSynchronize(ctx->stream));
    int64_t i = first, end = first + n;
    while (i < end) {
        const HostPop &p = ctx->pops[ctx->pop_of[i]];
        int64_t e = std::min(end, p.first + p.n);
        int64_t off = i - p.first, cnt = e - i;
        float *dst = buf + (i - first);
        if (p.kind == KIND_INPUT || var >= p.dev.nvars || !p.dev.x[var]) {
            if (get) std::fill(dst, dst + cnt, 0.0f);
            else if (p.kind != KIND_INPUT && var < p.dev.nvars) { set_error("state variable %d is not stored", var); return EB_ERR_ARG; }
        } else if (get) {
            CK(cudaMemcpy(dst, p.dev.x[var] + off, sizeof(float) * (size_t)cnt, cudaMemcpyDeviceToHost));
        } else {
            CK(cudaMemcpy(p.dev.x[var] + off, dst, sizeof(float) * (size_t)cnt, cudaMemcpyHostToDevice));
        }
        i = e;
    }
    return EB_OK;
}

int eb_get_state(eb_ctx *ctx, int64_t first, int64_t n, int var, float *out) {
    return state_io(ctx, first, n, var, out, true);
}
int eb_set_state(eb_ctx *ctx, int64_t first, int64_t n, int var, const float *in) {
    return state_io(ctx, first, n, var, const_cast<float *>(in), false);
}

int eb_set_trace(eb_ctx *ctx, int64_t first, int64_t n, int64_t steps) {
    if (!ctx || first < 0 || n < 0 || steps < 0 || first + n > ctx->n_neurons) { set_error("bad trace range"); return EB_ERR_ARG; }
    if (!ctx->finalized) { set_error("not finalized"); return EB_ERR_STATE; }
    size_t bytes = sizeof(float) * (size_t)n * (size_t)steps * kMaxVars;
    if (bytes > ctx->trace_bytes) {
        int rc = ctx->dalloc((void **)&ctx->net.trace, bytes);
        if (rc) return rc;
        ctx->trace_bytes = bytes;
    }
    if (bytes) CK(cudaMemsetAsync(ctx->net.trace, 0, bytes, ctx->stream));
    ctx->net.trace_first = first;
    ctx->net.trace_n = n;
    ctx->net.trace_steps = steps;
    ctx->trace_pending = true;
    ctx->graphs_valid = false;
    return EB_OK;
}

int eb_get_trace(eb_ctx *ctx, float *out) {
    if (!ctx || !out) { set_error("bad argument"); return EB_ERR_ARG; }
    CK(cudaStreamSynchronize(ctx->stream));
    size_t bytes = sizeof(float) * (size_t)ctx->net.trace_n * (size_t)ctx->net.trace_steps * kMaxVars;
    if (bytes) CK(cudaMemcpy(out, ctx->net.trace, bytes, cudaMemcpyDeviceToHost));
    return EB_OK;
}

int eb_get_weights(eb_ctx *ctx, float *w) {
    if (!ctx || !w) { set_error("bad argument"); return EB_ERR_ARG; }
    if (!ctx->finalized) { set_error("not finalized"); return EB_ERR_STATE; }
    int rc;
    if ((rc = ctx->flush_post())) return rc;  // deferred post-synaptic updates first
    CK(cudaStreamSynchronize(ctx->stream));
    const int64_t m = (int64_t)ctx->src.size();
    std::vector<SynRec> h(m);
    if (m) CK(cudaMemcpy(h.data(), ctx->net.syn, sizeof(SynRec) * (size_t)m, cudaMemcpyDeviceToHost));
    for (int64_t k = 0; k < m; ++k) w[k] = h[ctx->tpos_of[k]].w;
    return EB_OK;
}

int eb_set_weights(eb_ctx *ctx, const float *w) {
    if (!ctx || !w) { set_error("bad argument"); return EB_ERR_ARG; }
    if (!ctx->finalized) { set_error("not finalized"); return EB_ERR_STATE; }
    const int64_t m = (int64_t)ctx->src.size();
    std::vector<SynRec> h(m);
    int rc;
    if ((rc = ctx->flush_post())) return rc;  // pending post-synaptic updates belong to the old weights
    CK(cudaStreamSynchronize(ctx->stream));
    if (m) CK(cudaMemcpy(h.data(), ctx->net.syn, sizeof(SynRec) * (size_t)m, cudaMemcpyDeviceToHost));
    for (int64_t k = 0; k < m; ++k) h[ctx->tpos_of[k]].w = w[k];
    if (m) CK(cudaMemcpy(ctx->net.syn, h.data(), sizeof(SynRec) * (size_t)m, cudaMemcpyHostToDevice));
    return EB_OK;
}

int eb_set_random_seed(eb_ctx *ctx, uint32_t seed) {
    if (!ctx) { set_error("null context"); return EB_ERR_ARG; }
    if (ctx->finalized) { set_error("eb_set_random_seed after eb_finalize"); return EB_ERR_STATE; }
    ctx->rng_seed = seed;
    return EB_OK;
}

int eb_set_poisson_rates(eb_ctx *ctx, int64_t first, int64_t n, const float *rates_hz) {
    if (!ctx || n < 0 || (n > 0 && !rates_hz) || first < 0 || first + n > ctx->n_neurons) {
        set_error("eb_set_poisson_rates: bad argument");
        return EB_ERR_ARG;
    }
    for (auto &p : ctx->pops) {
        const int64_t lo = std::max(first, p.first), hi = std::min(first + n, p.first + p.n);
        if (lo >= hi) continue;
        if (p.kind != KIND_POISSON) {
            set_error("eb_set_poisson_rates: neurons %lld..%lld are not Poisson generators", (long long)lo, (long long)hi - 1);
            return EB_ERR_ARG;
        }
    }
    for (auto &p : ctx->pops) {
        const int64_t lo = std::max(first, p.first), hi = std::min(first + n, p.first + p.n);
        if (lo >= hi) continue;
        for (int64_t i = lo; i < hi; ++i) p.rates[i - p.first] = rates_hz[i - first];
        if (ctx->finalized) {
            std::vector<double> thr(hi - lo);
            for (int64_t i = lo; i < hi; ++i) thr[i - lo] = (double)p.rates[i - p.first] * (double)p.dt;
            CK(cudaStreamSynchronize(ctx->stream));
            CK(cudaMemcpy(const_cast<double *>(p.dev.pthr) + (lo - p.first), thr.data(), sizeof(double) * thr.size(),
                          cudaMemcpyHostToDevice));
        }
    }
    return EB_OK;
}

int eb_enable_conductances(eb_ctx *ctx, int pop, int mask) {
    if (!ctx) { set_error("null context"); return EB_ERR_ARG; }
    if (ctx->finalized) { set_error("eb_enable_conductances after eb_finalize"); return EB_ERR_STATE; }
    if (pop < 0 || pop >= (int)ctx->pops.size() || mask < 0 || mask > 7) { set_error("bad population or mask"); return EB_ERR_ARG; }
    ctx->pops[pop].en |= mask;
    return EB_OK;
}

int eb_population_state(eb_ctx *ctx, int pop, int var, float **device_ptr) {
    if (!ctx || !device_ptr) { set_error("bad argument"); return EB_ERR_ARG; }
    if (!ctx->finalized) { set_error("eb_population_state before eb_finalize"); return EB_ERR_STATE; }
    if (pop < 0 || pop >= (int)ctx->pops.size() || var < 0 || var >= kMaxVars) { set_error("bad population or variable"); return EB_ERR_ARG; }
    const auto &p = ctx->pops[pop];
    *device_ptr = (p.kind == KIND_INPUT || p.kind == KIND_POISSON || var >= p.dev.nvars) ? nullptr : p.dev.x[var];
    return EB_OK;
}

int eb_set_output(eb_ctx *ctx, int pop, int on) {
    if (!ctx) { set_error("null context"); return EB_ERR_ARG; }
    if (pop < 0 || pop >= (int)ctx->pops.size()) { set_error("population %d out of range", pop); return EB_ERR_ARG; }
    ctx->pops[pop].output = on != 0;
    return EB_OK;
}

int eb_set_monitor(eb_ctx *ctx, int pop, int on) {
    if (!ctx) { set_error("null context"); return EB_ERR_ARG; }
    if (pop < 0 || pop >= (int)ctx->pops.size()) { set_error("population %d out of range", pop); return EB_ERR_ARG; }
    ctx->pops[pop].monitor = on != 0;
    return EB_OK;
}

// The state monitor of the reference's -logp option: Simulation::WriteState
// (src/simulation/Simulation.cpp:397-405) into FileOutputSpikeDriver::WriteState
// (src/communication/FileOutputSpikeDriver.cpp:48-62) for the neurons of layers
// with the log column set (src/spike/Network.cpp:1102-1108).  The kernels keep
// each step's state of the monitored neurons and a log of the deliveries into
// them (weight and conductance type, in fold order); the host writes the lines
// after each chunk of steps.
int eb_open_monitor(eb_ctx *ctx, const char *path, int64_t chunk_steps, int64_t delivery_capacity) {
    if (!ctx || !path || chunk_steps < 0 || delivery_capacity < 0) { set_error("bad argument"); return EB_ERR_ARG; }
    if (!ctx->finalized) { set_error("eb_open_monitor before eb_finalize"); return EB_ERR_STATE; }
    int rc;
    if ((rc = ctx->close_monitor())) return rc;
    CK(cudaSetDevice(ctx->device));
    ctx->mon_cell.clear();
    ctx->mon_pop.clear();
    for (int q = 0; q < (int)ctx->pops.size(); ++q) {
        HostPop &p = ctx->pops[q];
        const bool on = p.monitor && (p.kind == KIND_LIF || p.kind == KIND_ADEX || p.kind == KIND_HH);
        p.dev.mon = on ? 1 : 0;
        p.dev.mon_base = on ? (int64_t)ctx->mon_cell.size() : 0;
        if (on)
            for (int64_t i = 0; i < p.n; ++i) {
                ctx->mon_cell.push_back(p.first + i);
                ctx->mon_pop.push_back(q);
            }
    }
    const int64_t n = (int64_t)ctx->mon_cell.size();
    const int64_t row = (int64_t)(sizeof(float) * kMaxVars + 1);
    const int64_t steps = chunk_steps ? chunk_steps
                                      : std::max<int64_t>(8, std::min<int64_t>(4096, (int64_t(64) << 20) / (row * std::max<int64_t>(n, 1))));
    const int64_t cap = delivery_capacity ? delivery_capacity : (int64_t(1) << 20);
    NetDev &N = ctx->net;
    if (n) {
        if ((rc = ctx->dalloc((void **)&N.mon_x, sizeof(float) * kMaxVars * (size_t)(steps * n))) ||
            (rc = ctx->dalloc((void **)&N.mon_spk, (size_t)(steps * n))) ||
            (rc = ctx->dalloc((void **)&N.mon_del, sizeof(MonDelivery) * (size_t)cap)) ||
            (rc = ctx->dalloc((void **)&N.mon_count, sizeof(unsigned long long)))) {
            ctx->close_monitor();
            return rc;
        }
        N.mon_n = n;
        N.mon_steps = steps;
        N.mon_cap = cap;
    }
    ctx->mon_file = std::fopen(path, "w");
    if (!ctx->mon_file) {
        ctx->close_monitor();
        set_error("cannot open %s for writing", path);
        return EB_ERR_ARG;
    }
    ctx->mon_steps = steps;
    ctx->mon_cap = cap;
    ctx->mon_cur.assign((size_t)n * kMaxVars, 0.0f);
    ctx->graphs_valid = false;
    ctx->pops_dirty = true;
    return EB_OK;
}

int eb_close_monitor(eb_ctx *ctx) {
    if (!ctx) { set_error("null context"); return EB_ERR_ARG; }
    return ctx->close_monitor();
}

int eb_ctx::close_monitor() {
    bool bad = false;
    if (mon_file) {
        bad = std::fclose(mon_file) != 0;
        mon_file = nullptr;
    }
    if (net.mon_x || net.mon_del) {
        CK(cudaStreamSynchronize(stream));
        dfree(net.mon_x);
        dfree(net.mon_spk);
        dfree(net.mon_del);
        dfree(net.mon_count);
    }
    net.mon_x = nullptr;
    net.mon_spk = nullptr;
    net.mon_del = nullptr;
    net.mon_count = nullptr;
    net.mon_n = net.mon_steps = net.mon_cap = 0;
    bool was_on = false;
    for (auto &p : pops) {
        was_on |= p.dev.mon != 0;
        p.dev.mon = 0;
        p.dev.mon_base = 0;
    }
    if (was_on) {
        graphs_valid = false;
        pops_dirty = true;
    }
    mon_cell.clear();
    mon_pop.clear();
    mon_cur.clear();
    if (bad) { set_error("write to the state monitor file failed"); return EB_ERR_ARG; }
    return EB_OK;
}

// eb_run with the monitor open: chunks of at most mon_steps steps, each followed
// by its lines.  The host copy of the monitored states starts every chunk from
// the device state, so states set between runs show up.
int eb_ctx::run_monitored(int64_t n) {
    const int64_t nm = (int64_t)mon_cell.size();
    std::vector<float> col;
    while (n > 0) {
        const int64_t c = std::min(n, mon_steps), k0 = steps_done;
        int rc;
        if (nm) {
            CK(cudaStreamSynchronize(stream));
            for (int64_t j = 0; j < nm;) {
                const HostPop &p = pops[mon_pop[j]];
                col.resize((size_t)p.n);
                for (int v = 0; v < kMaxVars; ++v) {
                    if (v < p.dev.nvars && p.dev.x[v])
                        CK(cudaMemcpy(col.data(), p.dev.x[v], sizeof(float) * (size_t)p.n, cudaMemcpyDeviceToHost));
                    else
                        std::fill(col.begin(), col.end(), 0.0f);
                    for (int64_t i = 0; i < p.n; ++i) mon_cur[(size_t)(j + i) * kMaxVars + v] = col[(size_t)i];
                }
                j += p.n;
            }
            CK(cudaMemsetAsync(net.mon_count, 0, sizeof(unsigned long long), stream));
        }
        if ((rc = run_async(c))) return rc;
        if ((rc = sync())) return rc;
        if (nm && (rc = write_monitor(k0, c))) return rc;
        n -= c;
    }
    return EB_OK;
}

// Lines of steps k0+1 .. k0+n: before each step's lines, the deliveries it folded
// in (time, synapse order), each after its weight is added to the host copy in
// that order (the device's float additions); then per monitored population the
// neurons that spiked and all its neurons, after the step.
int eb_ctx::write_monitor(int64_t k0, int64_t n) {
    const int64_t nm = (int64_t)mon_cell.size();
    unsigned long long cnt = 0;
    CK(cudaMemcpy(&cnt, net.mon_count, sizeof(cnt), cudaMemcpyDeviceToHost));
    if (cnt > (unsigned long long)mon_cap) { set_error("state monitor delivery log overflow"); return EB_ERR_OVERFLOW; }
    std::vector<MonDelivery> del((size_t)cnt);
    if (cnt) CK(cudaMemcpy(del.data(), net.mon_del, sizeof(MonDelivery) * (size_t)cnt, cudaMemcpyDeviceToHost));
    std::sort(del.begin(), del.end(), [](const MonDelivery &x, const MonDelivery &y) {
        if (x.k != y.k) return x.k < y.k;
        if (x.a != y.a) return x.a < y.a;
        if (x.spos != y.spos) return x.spos < y.spos;
        return x.cell < y.cell;
    });
    std::vector<float> xs((size_t)(mon_steps * nm) * kMaxVars);
    std::vector<uint8_t> sp((size_t)(mon_steps * nm));
    CK(cudaMemcpy(xs.data(), net.mon_x, sizeof(float) * xs.size(), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(sp.data(), net.mon_spk, sp.size(), cudaMemcpyDeviceToHost));
    std::FILE *f = mon_file;
    bool ok = true;
    auto line = [&](float t, int64_t j) {
        const HostPop &p = pops[mon_pop[j]];
        const float *x = &mon_cur[(size_t)j * kMaxVars];
        ok &= std::fprintf(f, "%f\t%li", (double)t, (long)mon_cell[j]) > 0;
        for (int v = 0; v < p.dev.nvars; ++v) ok &= std::fprintf(f, "\t%1.12f", (double)x[v]) > 0;
        // the reference's external-current variable (no current synapses on this
        // path), the last-update time a time-driven model never sets, and the two
        // event-driven fields a time-driven model prints as -1
        // (src/neuron_model/VectorNeuronState.cpp:193-209)
        ok &= std::fprintf(f, "\t%1.12f\t%1.12f\t%1.12f\t%1.12f\n", 0.0, 0.0, -1.0, -1.0) > 0;
    };
    size_t d = 0;
    while (d < del.size() && del[d].k <= k0) ++d;  // none expected
    for (int64_t k = k0 + 1; k <= k0 + n && ok; ++k) {
        for (; d < del.size() && del[d].k == k; ++d) {
            const MonDelivery &e = del[d];
            const int nd = pops[mon_pop[e.cell]].dev.ndiff;
            mon_cur[(size_t)e.cell * kMaxVars + nd + e.ty] += e.w;
            line((float)e.a, (int64_t)e.cell);
        }
        const int64_t row = k % mon_steps;
        std::copy(xs.begin() + (size_t)(row * nm) * kMaxVars, xs.begin() + (size_t)((row + 1) * nm) * kMaxVars,
                  mon_cur.begin());
        double t = 0.0;
        eb_step_time(this, k, &t);
        for (int64_t j = 0; j < nm;) {
            const int64_t e = j + pops[mon_pop[j]].n;
            for (int64_t i = j; i < e; ++i)
                if (sp[(size_t)(row * nm + i)]) line((float)t, i);
            for (int64_t i = j; i < e; ++i) line((float)t, i);
            j = e;
        }
    }
    if (!ok) { set_error("write to the state monitor file failed"); return EB_ERR_ARG; }
    return EB_OK;
}

// FileOutputSpikeDriver::WriteSpike (src/communication/FileOutputSpikeDriver.cpp:
// 40-46): one "%f\t%li" line per spike, the update time of its step and the
// neuron, for the neurons of populations with the output flag.
int eb_write_spikes(eb_ctx *ctx, const char *path, int append) {
    if (!ctx || !path) { set_error("bad argument"); return EB_ERR_ARG; }
    int64_t n = 0;
    int rc = eb_get_spikes(ctx, 0, &n, nullptr, nullptr);
    if (rc && rc != EB_ERR_OVERFLOW) return rc;
    std::vector<int64_t> st(n), ce(n);
    if (n && (rc = eb_get_spikes(ctx, n, &n, st.data(), ce.data()))) return rc;
    FILE *f = std::fopen(path, append ? "a" : "w");
    if (!f) { set_error("cannot open %s for writing", path); return EB_ERR_ARG; }
    for (int64_t i = 0; i < n; ++i) {
        if (!ctx->pops[ctx->pop_of[ce[i]]].output) continue;
        double t;
        eb_step_time(ctx, st[i], &t);
        if (std::fprintf(f, "%f\t%li\n", t, (long)ce[i]) < 0) {
            std::fclose(f);
            set_error("write to %s failed", path);
            return EB_ERR_ARG;
        }
    }
    if (std::fclose(f) != 0) { set_error("write to %s failed", path); return EB_ERR_ARG; }
    return EB_OK;
}

// Network::SaveWeights (src/spike/Network.cpp:1165-1202): the weights in
// network-file order as runs of equal values, one "%i %g" line per run.
int eb_save_weights(eb_ctx *ctx, const char *path) {
    if (!ctx || !path) { set_error("bad argument"); return EB_ERR_ARG; }
    const int64_t m = (int64_t)ctx->src.size();
    std::vector<float> w(m);
    int rc;
    if (m && (rc = eb_get_weights(ctx, w.data()))) return rc;
    FILE *f = std::fopen(path, "wt");
    if (!f) { set_error("cannot open %s for writing", path); return EB_ERR_ARG; }
    bool ok = true;
    for (int64_t i = 0; i < m && ok;) {
        const float v = w[i];
        int64_t j = i + 1;
        while (j < m && w[j] == v) ++j;
        ok = std::fprintf(f, "%i %g\n", (int)(j - i), (double)v) > 0;
        i = j;
    }
    if (std::fclose(f) != 0 || !ok) { set_error("write to %s failed", path); return EB_ERR_ARG; }
    return EB_OK;
}

int eb_get_population_events(eb_ctx *ctx, int pop, int64_t *events) {
    if (!ctx || !events) { set_error("null argument"); return EB_ERR_ARG; }
    if (!ctx->finalized) { set_error("not finalized"); return EB_ERR_STATE; }
    if (pop < 0 || pop >= (int)ctx->pops.size()) { set_error("population %d out of range", pop); return EB_ERR_ARG; }
    CK(cudaStreamSynchronize(ctx->stream));
    unsigned long long ev = 0;
    CK(cudaMemcpy(&ev, ctx->net.events + pop, sizeof(ev), cudaMemcpyDeviceToHost));
    *events = (int64_t)ev;
    return EB_OK;
}

int eb_get_counters(eb_ctx *ctx, int64_t *steps, int64_t *spikes, int64_t *events) {
    if (!ctx) { set_error("null context"); return EB_ERR_ARG; }
    if (!ctx->finalized) { set_error("not finalized"); return EB_ERR_STATE; }
    CK(cudaStreamSynchronize(ctx->stream));
    unsigned long long rc = 0;
    std::vector<unsigned long long> pe(ctx->pops.size());
    CK(cudaMemcpy(pe.data(), ctx->net.events, sizeof(unsigned long long) * pe.size(), cudaMemcpyDeviceToHost));
    unsigned long long ev = 0;
    for (auto v : pe) ev += v;
    CK(cudaMemcpy(&rc, ctx->net.rec_count, sizeof(rc), cudaMemcpyDeviceToHost));
    if (steps) *steps = ctx->steps_done;
    if (spikes) *spikes = ctx->spikes_drained + (int64_t)rc;
    if (events) *events = (int64_t)ev;
    return EB_OK;
}

int eb_snapshot(eb_ctx *ctx, int slot) {
    if (!ctx) { set_error("null context"); return EB_ERR_ARG; }
    return ctx->snapshot(slot);
}

int eb_restore(eb_ctx *ctx, int slot) {
    if (!ctx) { set_error("null context"); return EB_ERR_ARG; }
    return ctx->restore(slot);
}

int eb_stream(eb_ctx *ctx, void **stream) {
    if (!ctx || !stream) { set_error("bad argument"); return EB_ERR_ARG; }
    *stream = (void *)ctx->stream;
    return EB_OK;
}

int eb_prestage(eb_ctx *ctx, int64_t n_steps) {
    if (!ctx || n_steps < 0) { set_error("bad argument"); return EB_ERR_ARG; }
    if (!ctx->finalized) { set_error("not finalized"); return EB_ERR_STATE; }
    CK(cudaSetDevice(ctx->device));
    const int64_t k0 = ctx->steps_done, k_end = k0 + n_steps;
    int rc;
    if ((rc = ctx->ensure_tables(k_end + ctx->R + 8))) return rc;
    if ((rc = ctx->stage_inputs(k0, k_end))) return rc;
    CK(cudaStreamSynchronize(ctx->stream));
    return EB_OK;
}

int eb_set_profile(eb_ctx *ctx, int on) {
    if (!ctx) { set_error("null context"); return EB_ERR_ARG; }
    ctx->profile = on != 0;
    ctx->prof_sum.clear();
    return EB_OK;
}

int eb_get_profile(eb_ctx *ctx, int cap, int *n, int *kind, int *pop, int64_t *launches, double *total_ms) {
    if (!ctx || !n) { set_error("bad argument"); return EB_ERR_ARG; }
    int c = 0;
    for (auto &s : ctx->prof_sum) {
        if (c < cap) {
            if (kind) kind[c] = s.kind;
            if (pop) pop[c] = s.pop;
            if (launches) launches[c] = s.launches;
            if (total_ms) total_ms[c] = s.ms;
        }
        c++;
    }
    *n = c;
    return EB_OK;
}

int eb_launch_count(eb_ctx *ctx, int64_t *launches) {
    if (!ctx || !launches) { set_error("bad argument"); return EB_ERR_ARG; }
    *launches = ctx->launches;
    return EB_OK;
}

int eb_device_bytes(eb_ctx *ctx, int64_t *bytes) {
    if (!ctx || !bytes) { set_error("bad argument"); return EB_ERR_ARG; }
    *bytes = ctx->dev_bytes;
    return EB_OK;
}

}  // extern "C"
