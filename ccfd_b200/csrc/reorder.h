// Locality ordering of cells and faces for the device upload.
#pragma once

#include <vector>

#include "ccfd_b200.h"

// Reverse Cuthill-McKee order of the cell adjacency graph (device index ->
// reference cell) and a face order sorted by the lower device index of the
// two cells of each face (device index -> reference face).
void ccfd_rcm_order(const ccfd_mesh* m, std::vector<int>& cell_order, std::vector<int>& face_order);
