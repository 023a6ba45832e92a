// Test-infrastructure probe: dumps the lookup tables the reference CPU models
// build at run time (ExponentialTable, HH channel rates, LIF NMDA gating) so the
// restatements can be checked against the exact float values.
//   ref_tables out_prefix
#include <cstdio>
#include <string>
#include <map>
#include <any>
#define private public
#define protected public
#include "simulation/ExponentialTable.h"
#include "neuron_model/HHTimeDrivenModel.h"
#include "neuron_model/LIFTimeDrivenModel.h"
#undef private
#undef protected
int main(int argc, char **argv) {
    std::string out = argc > 1 ? argv[1] : "tables";
    FILE *f = std::fopen((out + ".exptable").c_str(), "wb");
    std::fwrite(ExponentialTable::LookUpTable, 4, ExponentialTable::TableSize, f);
    std::fclose(f);
    HHTimeDrivenModel hh;
    f = std::fopen((out + ".hhtable").c_str(), "wb");
    std::fwrite(hh.channel_values, 4, (size_t)HHTimeDrivenModel::TableSize * HHTimeDrivenModel::N_variables, f);
    std::fclose(f);
    LIFTimeDrivenModel lif;
    f = std::fopen((out + ".nmdatable").c_str(), "wb");
    std::fwrite(lif.g_nmda_inf_values, 4, LIFTimeDrivenModel::TableSizeNMDA, f);
    std::fclose(f);
    std::printf("ok %d %d %d\n", ExponentialTable::TableSize, HHTimeDrivenModel::TableSize, LIFTimeDrivenModel::TableSizeNMDA);
    return 0;
}
