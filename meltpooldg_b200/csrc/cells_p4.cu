// Cell kernels of FE_Q(4) (n = 5 points per direction).
#include "cells_degree.cuh"
MPDG_DEFINE_DEGREE(5)
