// Instantiates the batched modal sweep kernels (several problems per launch; see sweep_modal_impl.cuh).
#include "sweep_modal_impl.cuh"

IDC_MODAL_BATCHED(, 0)
IDC_MODAL_BATCHED(, 1)
