// Cell kernels of FE_Q(5) (n = 6 points per direction).
#include "cells_degree.cuh"
MPDG_DEFINE_DEGREE(6)
