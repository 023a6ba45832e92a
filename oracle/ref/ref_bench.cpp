// Timing driver for the reference EDLUT CPU kernel (built from the reference
// sources by oracle/ref/Makefile; test and benchmark infrastructure only).  It
// loads a network once through the reference's own Simulation class with Q
// OpenMP queues (the EDLUTKernel -openmp Q option, src/EDLUTKernel.cpp:93), runs
// a warm-up, then times `samples` consecutive samples of `sample_steps`
// integration steps each, one RunSimulationSlot call per sample
// (src/simulation/Simulation.cpp:322), with a monotonic wall clock.  Set-up
// (parsing, table building, InitSimulation) is timed separately and excluded.
//
// Usage: ref_bench net.cfg weights.cfg inputs.cfg|- queues dt_s warm_steps sample_steps samples
// Prints one JSON object on stdout.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <string>
#include <vector>
#include <list>
#include <map>
#include <any>

#include "simulation/Simulation.h"
#include "simulation/RandomGenerator.h"
#include "communication/FileInputSpikeDriver.h"
#include "spike/Network.h"
#include "openmp/openmp.h"

static double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

int main(int argc, char **argv) {
    if (argc < 9) {
        std::fprintf(stderr, "usage: %s net wts inputs|- queues dt warm_steps sample_steps samples\n", argv[0]);
        return 2;
    }
    const char *net = argv[1], *wts = argv[2], *inp = argv[3];
    int queues = std::atoi(argv[4]);
    const float dt = (float)std::atof(argv[5]);
    const long warm = std::atol(argv[6]), per = std::atol(argv[7]), samples = std::atol(argv[8]);
#ifdef _OPENMP
    if (queues > omp_get_max_threads()) queues = omp_get_max_threads();
#else
    queues = 1;
#endif
    if (queues < 1) queues = 1;
    RandomGenerator::srand(1);
    try {
        const double t_setup0 = now_s();
        const long total = warm + per * samples;
        const double T = ((double)total + 0.5) * (double)dt;
        Simulation sim(net, wts, T, 0.0, queues);
        if (std::strcmp(inp, "-") != 0) sim.AddInputSpikeDriver(new FileInputSpikeDriver(inp));
        sim.InitSimulation();
        const double setup = now_s() - t_setup0;
        // update times accumulate double(float(dt)) from 0, as the update event re-arms
        double t = 0.0;
        auto advance = [&](long steps) {
            for (long k = 0; k < steps; ++k) t += (double)dt;
            sim.RunSimulationSlot(t + 0.05 * (double)dt);
        };
        const double tw0 = now_s();
        if (warm > 0) advance(warm);
        const double warm_s = now_s() - tw0;
        std::vector<double> secs;
        std::vector<long long> spikes, events;
        long long s_prev = sim.GetTotalSpikeCounter(), e_prev = sim.GetTotalPropagateCounter();
        for (long i = 0; i < samples; ++i) {
            const double t0 = now_s();
            advance(per);
            secs.push_back(now_s() - t0);
            const long long s = sim.GetTotalSpikeCounter(), e = sim.GetTotalPropagateCounter();
            spikes.push_back(s - s_prev);
            events.push_back(e - e_prev);
            s_prev = s;
            e_prev = e;
        }
        std::printf("{\"queues\": %d, \"setup_s\": %.6f, \"warm_steps\": %ld, \"warm_s\": %.6f, "
                    "\"sample_steps\": %ld, \"neurons\": %d, \"sample_s\": [",
                    queues, setup, warm, warm_s, per, sim.GetNetwork()->GetNeuronNumber());
        for (size_t i = 0; i < secs.size(); ++i) std::printf("%s%.6f", i ? ", " : "", secs[i]);
        std::printf("], \"spikes\": [");
        for (size_t i = 0; i < spikes.size(); ++i) std::printf("%s%lld", i ? ", " : "", spikes[i]);
        std::printf("], \"events\": [");
        for (size_t i = 0; i < events.size(); ++i) std::printf("%s%lld", i ? ", " : "", events[i]);
        std::printf("]}\n");
    } catch (EDLUTException &e) {
        std::cerr << "EDLUT exception: " << e << std::endl;
        return 1;
    } catch (std::exception &e) {
        std::cerr << "exception: " << e.what() << std::endl;
        return 1;
    }
    return 0;
}
