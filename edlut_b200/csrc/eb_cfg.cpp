// Readers of the reference's text formats, so an existing EDLUT network runs
// unchanged:
//   network file   Network::ParseNet            src/spike/Network.cpp:422-645
//   weights file                                src/spike/Network.cpp:647-690
//   model .cfg     *TimeDrivenModel::ParseNeuronModel (e.g. LIFTimeDrivenModel.cpp:448-540),
//                  integration method           include/integration_method/IntegrationMethod.h:300-318,
//                                               BDFn.h:864-884
//   learning rule  STDPWeightChange::ParseLearningRule, src/learning_rules/STDPWeightChange.cpp:78-99
//   input spikes   FileInputSpikeDriver::LoadInputs, src/communication/FileInputSpikeDriver.cpp:45-78
// Comment and whitespace handling follows skip_comments / is_end_line
// (src/simulation/Utils.cpp).  Random weights (negative value in the weights
// file) use the reference's LCG (include/simulation/RandomGenerator.h:61-119)
// seeded like EDLUTKernel (RandomGenerator::srand(1), src/EDLUTKernel.cpp:88).
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "edlut_b200.h"
#include "eb_runtime.h"

using namespace eb;

namespace {

struct File {
    FILE *fh = nullptr;
    long line = 1;
    std::string name;
    explicit File(const std::string &n) : name(n) { fh = std::fopen(n.c_str(), "rt"); }
    ~File() { if (fh) std::fclose(fh); }
    int skip_spaces() {
        int ch;
        while ((ch = std::fgetc(fh)) == ' ' || ch == '\n')
            if (ch == '\n') line++;
        return ch;
    }
    void skip_comments() {
        int ch;
        while ((ch = skip_spaces()) == '/') {
            while ((ch = std::fgetc(fh)) != EOF && ch != '\n') {}
            if (ch == '\n') line++;
        }
        if (ch != EOF) std::ungetc(ch, fh);
    }
    bool is_end_line() {
        int ch;
        while ((ch = std::fgetc(fh)) == ' ') {}
        bool e = (ch == '\n' || ch == EOF || ch == '/');
        std::ungetc(ch, fh);
        return e;
    }
    int fail(const char *what) {
        set_error("%s:%ld: %s", name.c_str(), line, what);
        return EB_ERR_PARSE;
    }
};

// RandomGenerator of the reference: 31-bit LCG whose state is seeded from a seed
// chain -- each generator takes the chain's value, which then advances
// (RandomGenerator.cpp:21-27, include/simulation/RandomGenerator.h:61-68).  The
// reference keeps the chain in a process-global; here each load has its own, so
// contexts loading networks on different threads do not share it.
struct SeedChain {
    unsigned long seed;
    unsigned long take() {
        const unsigned long s = seed;
        seed = ((seed * 765426813) + 54321) & 0x7fffffff;
        return s;
    }
};
struct RefRandom {
    unsigned long next;
    explicit RefRandom(SeedChain &chain) : next(chain.take()) {}
    float frand() {
        next = ((next * 1103515245) + 12345) & 0x7fffffff;
        return ((float)next) / 2147483647;
    }
};

const char *kModelNames[] = {"InputSpikeNeuronModel", "LIFTimeDrivenModel", "AdExTimeDrivenModel",
                             "HHTimeDrivenModel", "PoissonGeneratorDeviceVector"};
const int kModelParams[] = {0, 10, 14, 13, 1};

int model_kind(const std::string &name) {
    for (int k = 0; k < 5; ++k) {
        std::string n = kModelNames[k];
        if (name == n || (k > 0 && k < 4 && name == n + "_GPU")) return k;
    }
    return -1;
}

int parse_model_cfg(const std::string &path, int kind, std::vector<float> &params, int &integ, int &order,
                    float &dt) {
    File f(path);
    if (!f.fh) { set_error("cannot open neuron model file %s", path.c_str()); return EB_ERR_PARSE; }
    params.clear();
    for (int i = 0; i < kModelParams[kind]; ++i) {
        f.skip_comments();
        float v;
        if (std::fscanf(f.fh, "%f", &v) != 1) return f.fail("missing neuron model parameter");
        params.push_back(v);
    }
    if (kind == KIND_POISSON) {  // PoissonGeneratorDeviceVector::ParseNeuronModel: the frequency only
        integ = 0;
        order = 0;
        dt = 0.1f / 1000.0f;
        return EB_OK;
    }
    f.skip_comments();
    char name[65];
    if (std::fscanf(f.fh, "%64s", name) != 1) return f.fail("missing integration method");
    std::string in = name;
    order = 0;
    if (in == "Euler") integ = INTEG_EULER;
    else if (in == "RK2") integ = INTEG_RK2;
    else if (in == "RK4") integ = INTEG_RK4;
    else if (in == "BDF") {
        integ = INTEG_BDF;
        f.skip_comments();
        if (std::fscanf(f.fh, "%d", &order) != 1) return f.fail("missing BDF order");
        if (order < 1 || order > 6) return f.fail("BDF order must be 1..6");
    } else {
        set_error("%s: integration method %s is outside this path (Euler, RK2, RK4, BDF)", path.c_str(), name);
        return EB_ERR_UNSUPPORTED;
    }
    f.skip_comments();
    if (std::fscanf(f.fh, "%f", &dt) != 1 || !(dt > 0.0f)) return f.fail("missing or bad integration step");
    return EB_OK;
}

}  // namespace

extern "C" int eb_load_network_files(eb_ctx *ctx, const char *network_file, const char *weights_file) {
    if (!ctx || !network_file || !weights_file) { set_error("null argument"); return EB_ERR_ARG; }
    if (ctx->finalized || ctx->n_neurons) { set_error("eb_load_network_files on a non-empty context"); return EB_ERR_STATE; }
    File f(network_file);
    if (!f.fh) { set_error("cannot open network file %s", network_file); return EB_ERR_PARSE; }
    int ntypes = 0, nneurons = 0;
    f.skip_comments();
    if (std::fscanf(f.fh, "%i", &ntypes) != 1 || ntypes <= 0) return f.fail("bad number of neuron types");
    f.skip_comments();
    if (std::fscanf(f.fh, "%i", &nneurons) != 1 || nneurons <= 0) return f.fail("bad number of neurons");
    int rc;
    for (int done = 0, nn = 0; done < nneurons; done += nn) {
        f.skip_comments();
        char type[65], ident[65];
        int outn, monit;
        if (std::fscanf(f.fh, "%i", &nn) != 1 || nn <= 0 || std::fscanf(f.fh, "%64s", type) != 1 ||
            std::fscanf(f.fh, "%64s", ident) != 1 || std::fscanf(f.fh, "%i", &outn) != 1 ||
            std::fscanf(f.fh, "%i", &monit) != 1)
            return f.fail("bad neuron layer line");
        if (done + nn > nneurons) return f.fail("layers exceed the number of neurons");
        int kind = model_kind(type);
        if (kind < 0) {
            set_error("%s:%ld: neuron model %s is outside this path", network_file, f.line, type);
            return EB_ERR_UNSUPPORTED;
        }
        if (kind == KIND_INPUT) {
            if ((rc = ctx->add_population(KIND_INPUT, nn, 0, 0, 0.0f, nullptr, 0, nullptr))) return rc;
        } else {
            std::vector<float> params;
            int integ = 0, order = 0;
            float dt = 0;
            if ((rc = parse_model_cfg(std::string(ident) + ".cfg", kind, params, integ, order, dt))) return rc;
            if ((rc = ctx->add_population(kind, nn, integ, order, dt, params.data(), (int)params.size(), nullptr)))
                return rc;
        }
        ctx->pops.back().output = outn != 0;
        ctx->pops.back().monitor = monit != 0 && kind != KIND_INPUT;
    }
    f.skip_comments();
    int nrules = 0;
    if (std::fscanf(f.fh, "%i", &nrules) != 1 || nrules < 0) return f.fail("bad number of learning rules");
    for (int r = 0; r < nrules; ++r) {
        f.skip_comments();
        char name[65];
        if (std::fscanf(f.fh, "%64s", name) != 1) return f.fail("missing learning rule");
        if (std::string(name) != "STDP") {
            set_error("%s:%ld: learning rule %s is outside this path (STDP only)", network_file, f.line, name);
            return EB_ERR_UNSUPPORTED;
        }
        float p[4];
        for (int i = 0; i < 4; ++i)
            if (std::fscanf(f.fh, "%f", &p[i]) != 1) return f.fail("bad STDP parameters");
        if (p[1] <= 0 || p[3] <= 0) return f.fail("STDP time constants must be > 0");
        ctx->rules.push_back({p[0], p[1], p[2], p[3]});
    }
    f.skip_comments();
    long ninters = 0;
    if (std::fscanf(f.fh, "%li", &ninters) != 1 || ninters <= 0) return f.fail("bad number of synapses");
    std::vector<int64_t> src(ninters), tgt(ninters);
    std::vector<float> dly(ninters, 0.001f), maxw(ninters, 1.0f), w(ninters, 1.0f);
    std::vector<int32_t> typ(ninters, 0), rule(ninters, -1);
    for (long i = 0; i < ninters;) {
        f.skip_comments();
        int s, ns, t, nt, nr, type, wc1 = -1, wc2 = -1;
        float d, dinc, mw;
        if (std::fscanf(f.fh, "%i", &s) != 1 || std::fscanf(f.fh, "%i", &ns) != 1 || std::fscanf(f.fh, "%i", &t) != 1 ||
            std::fscanf(f.fh, "%i", &nt) != 1 || std::fscanf(f.fh, "%i", &nr) != 1 || std::fscanf(f.fh, "%f", &d) != 1 ||
            std::fscanf(f.fh, "%f", &dinc) != 1 || std::fscanf(f.fh, "%i", &type) != 1 || std::fscanf(f.fh, "%f", &mw) != 1)
            return f.fail("bad synapse line");
        bool trig1 = false;
        if (std::fscanf(f.fh, " t%d", &wc1) == 1) trig1 = true;
        else if (std::fscanf(f.fh, "%d", &wc1) != 1) return f.fail("missing learning rule index");
        if (wc1 >= nrules) return f.fail("learning rule index out of range");
        if (wc1 >= 0 && !f.is_end_line()) {
            if (std::fscanf(f.fh, " t%d", &wc2) == 1 || std::fscanf(f.fh, "%d", &wc2) == 1) {
                set_error("%s:%ld: trigger learning rules are outside this path", network_file, f.line);
                return EB_ERR_UNSUPPORTED;
            }
        }
        if (trig1 && wc1 >= 0) {
            set_error("%s:%ld: trigger learning rules are outside this path", network_file, f.line);
            return EB_ERR_UNSUPPORTED;
        }
        if (ns <= 0 || nt <= 0 || nr <= 0) return f.fail("bad synapse block sizes");
        if (i + (long)ns * nt * nr > ninters) return f.fail("synapse blocks exceed the number of synapses");
        for (int r = 0; r < nr; ++r)
            for (int a = 0; a < ns; ++a)
                for (int b = 0; b < nt; ++b) {
                    long pos = i + (long)r * ns * nt + (long)a * nt + b;
                    src[pos] = s + (long)r * ns + a;
                    tgt[pos] = t + (long)r * nt + b;
                    dly[pos] = d + dinc * b;
                    typ[pos] = type;
                    maxw[pos] = mw;
                    rule[pos] = wc1;
                }
        i += (long)ns * nt * nr;
    }
    // weights file
    File g(weights_file);
    if (!g.fh) { set_error("cannot open weights file %s", weights_file); return EB_ERR_PARSE; }
    SeedChain chain{ctx->rng_seed & 0x7fffffffu};
    RefRandom rnd(chain);
    g.skip_comments();
    for (long c = 0; c < ninters;) {
        g.skip_comments();
        int nw;
        float wv;
        if (std::fscanf(g.fh, "%i", &nw) != 1 || std::fscanf(g.fh, "%f", &wv) != 1) return g.fail("bad weight line");
        if (nw < 0 || nw + c > ninters) return g.fail("weights exceed the number of synapses");
        if (nw == 0) nw = (int)(ninters - c);
        for (int k = 0; k < nw; ++k) {
            double cw;
            if (wv < 0.0f) cw = rnd.frand() * maxw[c + k];
            else if (wv > maxw[c + k]) cw = maxw[c + k];
            else cw = wv;
            w[c + k] = (float)cw;
        }
        c += nw;
    }
    ctx->src.swap(src);
    ctx->tgt.swap(tgt);
    ctx->delay.swap(dly);
    ctx->stype.swap(typ);
    ctx->weight.swap(w);
    ctx->max_weight.swap(maxw);
    ctx->rule.swap(rule);
    return ctx->finalize(nullptr);
}

extern "C" int eb_load_input_file(eb_ctx *ctx, const char *input_file) {
    if (!ctx || !input_file) { set_error("null argument"); return EB_ERR_ARG; }
    File f(input_file);
    if (!f.fh) { set_error("cannot open input file %s", input_file); return EB_ERR_PARSE; }
    f.skip_comments();
    int ninputs = 0;
    if (std::fscanf(f.fh, "%i", &ninputs) != 1) return f.fail("bad number of input spikes");
    std::vector<float> times;
    std::vector<int64_t> cells;
    for (int i = 0; i < ninputs;) {
        f.skip_comments();
        float time, interv;
        int nspikes, nneuron, nreps;
        if (std::fscanf(f.fh, "%f", &time) != 1 || std::fscanf(f.fh, "%i", &nspikes) != 1 ||
            std::fscanf(f.fh, "%f", &interv) != 1 || std::fscanf(f.fh, "%i", &nneuron) != 1 ||
            std::fscanf(f.fh, "%i", &nreps) != 1)
            return f.fail("too few input spikes");
        if (nneuron < 0 || nneuron + nreps > ctx->n_neurons) return f.fail("input neuron out of range");
        i += nspikes * nreps;
        if (i > ninputs) return f.fail("more input spikes than declared");
        for (int s = 0; s < nspikes; ++s)
            for (int r = 0; r < nreps; ++r) {
                times.push_back(time + s * interv);
                cells.push_back(nneuron + r);
            }
    }
    return eb_inject_spikes(ctx, (int64_t)times.size(), times.data(), cells.data());
}
