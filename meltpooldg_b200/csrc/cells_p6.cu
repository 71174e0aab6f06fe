// Cell kernels of FE_Q(6) (n = 7 points per direction).
#include "cells_degree.cuh"
MPDG_DEFINE_DEGREE(7)
