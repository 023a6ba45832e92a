// Test-infrastructure driver for the reference EDLUT CPU kernel (built from the
// reference sources by oracle/ref/Makefile).  It runs a network file through the
// reference's own Simulation class, one neuron-update step at a time, and dumps
// binary records that the golden-fixture generator turns into test vectors:
//
//   <out>.spikes   int64 n, then n x {double time, int64 cell}     (output order)
//   <out>.trace    int32 steps, int32 ncells, int32 nvars, then per step per
//                  cell nvars float32 state variables (state AFTER the update)
//   <out>.syn      int64 m, then m x {int64 orig_index, int64 source, int64 target,
//                  double delay, int32 type, float weight_final}   in the
//                  reference's sorted synapse order (qsort_inters, Network.cpp:45-68)
//   <out>.wfinal   int64 m, then m float32 final weights in network-file order
//   <out>.counts   text: spikes propagated_events
//   <out>.of       text: the reference's own FileOutputSpikeDriver file (-of)
//   <out>.logp     text: the reference's own state monitor file (-logp), the states
//                  of the neurons of layers whose log column is set, every step
//   <out>.sf       text: the reference's own Network::SaveWeights file (-sf)
//
// Usage: ref_harness net.cfg weights.cfg inputs.cfg|- nsteps dt_s out_prefix
//                    [trace_steps trace_first_cell trace_ncells]
//
// The step loop mirrors EDLUTKernel's RunSimulation by slots: RunSimulationSlot
// (Simulation.cpp:322) is called with a preempt time half a tenth of a step
// after each update time (just after the last one), so the event order inside a
// step is the reference's.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cstdint>
#include <vector>
#include <string>
#include <iostream>
#include <fstream>
#include <list>
#include <map>
#include <any>

#define private public
#define protected public
#include "simulation/Simulation.h"
#include "simulation/RandomGenerator.h"
#include "spike/Network.h"
#include "spike/Neuron.h"
#include "spike/Interconnection.h"
#include "neuron_model/VectorNeuronState.h"
#include "neuron_model/NeuronModel.h"
#include "communication/FileInputSpikeDriver.h"
#include "communication/ArrayOutputSpikeDriver.h"
#include "communication/FileOutputSpikeDriver.h"
#undef private
#undef protected

int main(int argc, char **argv) {
    if (argc < 7) {
        std::fprintf(stderr, "usage: %s net wts inputs|- nsteps dt out [trace_steps first ncells]\n", argv[0]);
        return 2;
    }
    const char *net = argv[1], *wts = argv[2], *inp = argv[3];
    long nsteps = std::atol(argv[4]);
    float dt = (float)std::atof(argv[5]);
    std::string out = argv[6];
    long trace_steps = argc > 7 ? std::atol(argv[7]) : 0;
    long trace_first = argc > 8 ? std::atol(argv[8]) : 0;
    long trace_n = argc > 9 ? std::atol(argv[9]) : 0;

    RandomGenerator::srand(1);
    try {
        double T = ((double)nsteps + 0.5) * (double)dt;
        Simulation sim(net, wts, T, 0.0, 1);
        if (std::strcmp(inp, "-") != 0) sim.AddInputSpikeDriver(new FileInputSpikeDriver(inp));
        ArrayOutputSpikeDriver *outdrv = new ArrayOutputSpikeDriver();
        sim.AddOutputSpikeDriver(outdrv);
        FileOutputSpikeDriver *filedrv = new FileOutputSpikeDriver((out + ".of").c_str(), false);
        sim.AddOutputSpikeDriver(filedrv);
        FileOutputSpikeDriver *logdrv = new FileOutputSpikeDriver((out + ".logp").c_str(), true);
        sim.AddMonitorActivityDriver(logdrv);
        sim.InitSimulation();

        Network *nw = sim.GetNetwork();
        int nvars = 0;
        if (trace_n > 0) nvars = nw->GetNeuronAt(trace_first)->GetVectorNeuronState()->GetNumberOfVariables();
        FILE *ft = nullptr;
        if (trace_n > 0) {
            ft = std::fopen((out + ".trace").c_str(), "wb");
            int32_t h[3] = {(int32_t)trace_steps, (int32_t)trace_n, (int32_t)nvars};
            std::fwrite(h, sizeof(h), 1, ft);
        }
        std::vector<double> st;
        std::vector<int64_t> sc;
        double t = 0.0;
        for (long k = 1; k <= nsteps; ++k) {
            t += (double)dt;  // the update event re-arms at CurrentTime + step (TimeEventUpdateNeurons.cpp:115)
            // after the last update stop before any later delivery (arrivals trail an
            // update time by at least ~1e-12 s), so final weights carry no partial step
            sim.RunSimulationSlot(k == nsteps ? t + 1e-13 : t + 0.05 * (double)dt);
            if (ft && k <= trace_steps) {
                for (long c = trace_first; c < trace_first + trace_n; ++c) {
                    Neuron *n = nw->GetNeuronAt(c);
                    VectorNeuronState *vs = n->GetVectorNeuronState();
                    for (int v = 0; v < nvars; ++v) {
                        float x = vs->GetStateVariableAt(n->GetIndex_VectorNeuronState(), v);
                        std::fwrite(&x, 4, 1, ft);
                    }
                }
            }
            double *times; long int *cells;
            unsigned int ns = outdrv->GetBufferedSpikes(times, cells);
            for (unsigned int i = 0; i < ns; ++i) { st.push_back(times[i]); sc.push_back(cells[i]); }
            if (ns > 0) { delete[] times; delete[] cells; }
        }
        if (ft) std::fclose(ft);

        FILE *fs = std::fopen((out + ".spikes").c_str(), "wb");
        int64_t n = (int64_t)st.size();
        std::fwrite(&n, 8, 1, fs);
        for (int64_t i = 0; i < n; ++i) { std::fwrite(&st[i], 8, 1, fs); std::fwrite(&sc[i], 8, 1, fs); }
        std::fclose(fs);

        FILE *fy = std::fopen((out + ".syn").c_str(), "wb");
        int64_t m = nw->ninters;
        std::fwrite(&m, 8, 1, fy);
        for (int64_t j = 0; j < m; ++j) {
            Interconnection &ic = nw->inters[j];
            int64_t oi = ic.GetIndex(), s = ic.GetSource()->GetIndex(), tg = ic.GetTarget()->GetIndex();
            double d = ic.GetDelay();
            int32_t ty = ic.GetType();
            float w = ic.GetWeight();
            std::fwrite(&oi, 8, 1, fy); std::fwrite(&s, 8, 1, fy); std::fwrite(&tg, 8, 1, fy);
            std::fwrite(&d, 8, 1, fy); std::fwrite(&ty, 4, 1, fy); std::fwrite(&w, 4, 1, fy);
        }
        std::fclose(fy);

        FILE *fw = std::fopen((out + ".wfinal").c_str(), "wb");
        std::fwrite(&m, 8, 1, fw);
        for (int64_t j = 0; j < m; ++j) { float w = nw->wordination[j]->GetWeight(); std::fwrite(&w, 4, 1, fw); }
        std::fclose(fw);

        nw->SaveWeights((out + ".sf").c_str());
        std::fflush(filedrv->Handler);
        std::fflush(logdrv->Handler);

        std::ofstream fc(out + ".counts");
        fc << sim.GetTotalSpikeCounter() << " " << sim.GetTotalPropagateCounter() << "\n";
    } catch (EDLUTException &e) {
        std::cerr << "EDLUT exception: " << e << std::endl;
        return 1;
    } catch (std::exception &e) {
        std::cerr << "exception: " << e.what() << std::endl;
        return 1;
    }
    return 0;
}
