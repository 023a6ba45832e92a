// The reference's neuron-model factory (the NeuronModelFactory class declared in
// include/neuron_model/NeuronModelFactory.h) for a GPU build of the reference
// engine whose LIFTimeDrivenModel_GPU, AdExTimeDrivenModel_GPU and
// HHTimeDrivenModel_GPU names create the libedlut_b200 plugins (b200_models.cu).
// It takes the place of src/neuron_model/NeuronModelFactory.cu in that build: the
// same registry (model name -> parse, create, default-parameter, information and
// vectorizable-parameter functions, src/neuron_model/NeuronModelFactory.cu:85-257)
// and the same lookups and errors; every other model keeps the reference's own
// functions.
#include <iostream>
#include <map>
#include <string>
#include <type_traits>
#include <vector>
#include <any>

#include "neuron_model/NeuronModelFactory.h"
#include "neuron_model/NeuronModel.h"
#include "neuron_model/InputCurrentNeuronModel.h"
#include "neuron_model/InputSpikeNeuronModel.h"
#include "neuron_model/PoissonGeneratorDeviceVector.h"
#include "neuron_model/SinCurrentDeviceVector.h"
#include "neuron_model/AdExTimeDrivenModel.h"
#include "neuron_model/AdExTimeDrivenModelVector.h"
#include "neuron_model/EgidioGranuleCell_TimeDriven.h"
#include "neuron_model/HHTimeDrivenModel.h"
#include "neuron_model/IzhikevichTimeDrivenModel.h"
#include "neuron_model/LIFTimeDrivenModel.h"
#include "neuron_model/LIFTimeDrivenModel_IS.h"
#include "neuron_model/TimeDrivenInferiorOliveCell.h"
#include "neuron_model/TimeDrivenPurkinjeCell.h"
#include "neuron_model/TimeDrivenPurkinjeCell_IP.h"
#include "neuron_model/CompressSynchronousTableBasedModel.h"
#include "neuron_model/CompressTableBasedModel.h"
#include "neuron_model/SynchronousTableBasedModel.h"
#include "neuron_model/TableBasedModel.h"
#include "neuron_model/AdExTimeDrivenModel_GPU_C_INTERFACE.cuh"
#include "neuron_model/EgidioGranuleCell_TimeDriven_GPU_C_INTERFACE.cuh"
#include "neuron_model/HHTimeDrivenModel_GPU_C_INTERFACE.cuh"
#include "neuron_model/IzhikevichTimeDrivenModel_GPU_C_INTERFACE.cuh"
#include "neuron_model/LIFTimeDrivenModel_GPU_C_INTERFACE.cuh"
#include "neuron_model/LIFTimeDrivenModel_IS_GPU_C_INTERFACE.cuh"
#include "neuron_model/TimeDrivenPurkinjeCell_GPU_C_INTERFACE.cuh"
#include "spike/EDLUTException.h"

#include "b200_models.h"

std::map<std::string, NeuronModelFactory::NeuronModelClass> NeuronModelFactory::NeuronModelMap;

void NeuronModelFactory::InitializeNeuronModelFactory() {
    if (!NeuronModelMap.empty()) return;
    // a model class's own static functions under its own name
    auto add = [](auto *tag) {
        using M = std::remove_pointer_t<decltype(tag)>;
        NeuronModelMap[M::GetName()] =
            NeuronModelClass(M::ParseNeuronModel, M::CreateNeuronModel, M::GetDefaultParameters, M::GetNeuronModelInfo);
    };
    auto add_vector = [](auto *tag) {
        using M = std::remove_pointer_t<decltype(tag)>;
        NeuronModelMap[M::GetName()] = NeuronModelClass(M::ParseNeuronModel, M::CreateNeuronModel, M::GetDefaultParameters,
                                                        M::GetNeuronModelInfo, M::GetVectorizableParameters);
    };
    // the reference's .cfg parsing, defaults and information, this library's model
    auto add_b200 = [](auto *tag, CreateNeuronModelFunc create) {
        using M = std::remove_pointer_t<decltype(tag)>;
        NeuronModelMap[M::GetName()] =
            NeuronModelClass(M::ParseNeuronModel, create, M::GetDefaultParameters, M::GetNeuronModelInfo);
    };
    add((InputCurrentNeuronModel *)nullptr);
    add((InputSpikeNeuronModel *)nullptr);
    add_vector((PoissonGeneratorDeviceVector *)nullptr);
    add_vector((SinCurrentDeviceVector *)nullptr);
    add((AdExTimeDrivenModel *)nullptr);
    add_vector((AdExTimeDrivenModelVector *)nullptr);
    add((EgidioGranuleCell_TimeDriven *)nullptr);
    add((HHTimeDrivenModel *)nullptr);
    add((IzhikevichTimeDrivenModel *)nullptr);
    add((LIFTimeDrivenModel *)nullptr);
    add((LIFTimeDrivenModel_IS *)nullptr);
    add((TimeDrivenInferiorOliveCell *)nullptr);
    add((TimeDrivenPurkinjeCell *)nullptr);
    add((TimeDrivenPurkinjeCell_IP *)nullptr);
    add((CompressSynchronousTableBasedModel *)nullptr);
    add((CompressTableBasedModel *)nullptr);
    add((SynchronousTableBasedModel *)nullptr);
    add((TableBasedModel *)nullptr);
    add((EgidioGranuleCell_TimeDriven_GPU_C_INTERFACE *)nullptr);
    add((IzhikevichTimeDrivenModel_GPU_C_INTERFACE *)nullptr);
    add((LIFTimeDrivenModel_IS_GPU_C_INTERFACE *)nullptr);
    add((TimeDrivenPurkinjeCell_GPU_C_INTERFACE *)nullptr);
    add_b200((LIFTimeDrivenModel_GPU_C_INTERFACE *)nullptr, b200_create_lif);
    add_b200((AdExTimeDrivenModel_GPU_C_INTERFACE *)nullptr, b200_create_adex);
    add_b200((HHTimeDrivenModel_GPU_C_INTERFACE *)nullptr, b200_create_hh);
}

namespace {
// The registry entry of a model name; the reference's error for unknown names.
template <class Map>
typename Map::const_iterator find_model(const Map &m, const std::string &ident) {
    auto it = m.find(ident);
    if (it == m.end())
        throw EDLUTException(TASK_NETWORK_LOAD_NEURON_MODELS, ERROR_NETWORK_NEURON_MODEL_TYPE,
                             REPAIR_NETWORK_NEURON_MODEL_TYPE);
    return it;
}

void print_entries(const std::string &ident, const std::map<std::string, std::string> &m) {
    auto info = m.find("info");
    if (info != m.end()) std::cout << "\t- " << ident << ": " << info->second << std::endl;
    for (const auto &kv : m)
        if (kv.first != "info") std::cout << "\t\t- " << kv.first << ": " << kv.second << std::endl;
}
}  // namespace

std::vector<std::string> NeuronModelFactory::GetAvailableNeuronModels() {
    InitializeNeuronModelFactory();
    std::vector<std::string> names;
    for (const auto &kv : NeuronModelMap) names.push_back(kv.first);
    return names;
}

void NeuronModelFactory::PrintAvailableNeuronModels() {
    std::cout << "- Available Neuron Models in EDLUT:" << std::endl;
    for (const std::string &n : GetAvailableNeuronModels()) std::cout << "\t- " << n << std::endl;
}

NeuronModel *NeuronModelFactory::CreateNeuronModel(ModelDescription desc) noexcept(false) {
    InitializeNeuronModelFactory();
    return find_model(NeuronModelMap, desc.model_name)->second.createFunc(desc);
}

ModelDescription NeuronModelFactory::ParseNeuronModel(std::string ident, std::string ident_param) noexcept(false) {
    InitializeNeuronModelFactory();
    if (NeuronModelMap.find(ident) == NeuronModelMap.end())
        std::cout << "Neuron model \"" << ident << "\" does not exist" << std::endl;
    return find_model(NeuronModelMap, ident)->second.parseFunc(ident_param + std::string(".cfg"));
}

std::map<std::string, boost::any> NeuronModelFactory::GetDefaultParameters(std::string ident) noexcept(false) {
    InitializeNeuronModelFactory();
    return find_model(NeuronModelMap, ident)->second.getDefaultParamFunc();
}

std::map<std::string, std::string> NeuronModelFactory::GetNeuronModelInfo(std::string ident) noexcept(false) {
    InitializeNeuronModelFactory();
    return find_model(NeuronModelMap, ident)->second.getInfoFunc();
}

void NeuronModelFactory::PrintNeuronModelInfo(std::string ident) noexcept(false) {
    const std::map<std::string, std::string> m = GetNeuronModelInfo(ident);
    std::cout << "- Information about neuron model " << ident << std::endl;
    print_entries(ident, m);
}

std::map<std::string, std::string> NeuronModelFactory::GetVectorizableParameters(std::string ident) noexcept(false) {
    InitializeNeuronModelFactory();
    return find_model(NeuronModelMap, ident)->second.getVectorizableParamFunc();
}

void NeuronModelFactory::PrintVectorizableParameters(std::string ident) noexcept(false) {
    const std::map<std::string, std::string> m = GetVectorizableParameters(ident);
    std::cout << "- Vectorizable parameters of neuron model " << ident << std::endl;
    print_entries(ident, m);
}
