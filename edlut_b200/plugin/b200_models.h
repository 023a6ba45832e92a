// Creation functions of the libedlut_b200 neuron-model plugins (b200_models.cu),
// in the form the reference's model factory stores (CreateNeuronModelFunc,
// include/neuron_model/NeuronModelFactory.h:51).
#pragma once
#include "simulation/NetworkDescription.h"

class NeuronModel;

NeuronModel *b200_create_lif(ModelDescription d);
NeuronModel *b200_create_adex(ModelDescription d);
NeuronModel *b200_create_hh(ModelDescription d);
