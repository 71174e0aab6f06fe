// Cell kernels of FE_Q(1) (n = 2 points per direction).
#include "cells_degree.cuh"
MPDG_DEFINE_DEGREE(2)
