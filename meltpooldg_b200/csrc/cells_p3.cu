// Cell kernels of FE_Q(3) (n = 4 points per direction).
#include "cells_degree.cuh"
MPDG_DEFINE_DEGREE(4)
