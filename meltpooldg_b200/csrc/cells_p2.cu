// Cell kernels of FE_Q(2) (n = 3 points per direction).
#include "cells_degree.cuh"
MPDG_DEFINE_DEGREE(3)
