// Instantiates the modal sweep kernels of one precision (see sweep_modal_impl.cuh).
#include "sweep_modal_impl.cuh"

IDC_MODAL_LAUNCHERS(, 1, false)
IDC_MODAL_LAUNCHERS(, 1, true)
