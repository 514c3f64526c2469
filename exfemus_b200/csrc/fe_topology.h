// fe_topology.h -- element topology shared by host and device code.
//
// libMesh Quad9/Hex27 local node order, as used by the reference's shape functions
// (src/MGFE.C:195-370) and surface topology _surf_top (include/MGGeomEl.h:39-51,
// src/MGGeomEl.C:172-177 and :310-317).  Each local node is given by its lattice
// offset (a,b,c) in half-element units; a side lists its nodes with the midpoint/centre
// last, which the assembly uses to decide whether the side is Dirichlet.
#pragma once

namespace exf {

constexpr int Q9_ABC[9][3] = {{0, 0, 0}, {2, 0, 0}, {2, 2, 0}, {0, 2, 0}, {1, 0, 0},
                              {2, 1, 0}, {1, 2, 0}, {0, 1, 0}, {1, 1, 0}};
constexpr int H27_ABC[27][3] = {
    {0, 0, 0}, {2, 0, 0}, {2, 2, 0}, {0, 2, 0}, {0, 0, 2}, {2, 0, 2}, {2, 2, 2}, {0, 2, 2},
    {1, 0, 0}, {2, 1, 0}, {1, 2, 0}, {0, 1, 0}, {0, 0, 1}, {2, 0, 1}, {2, 2, 1}, {0, 2, 1},
    {1, 0, 2}, {2, 1, 2}, {1, 2, 2}, {0, 1, 2}, {1, 1, 0}, {1, 0, 1}, {2, 1, 1}, {1, 2, 1},
    {0, 1, 1}, {1, 1, 2}, {1, 1, 1}};
constexpr int Q9_SIDE[4][3] = {{0, 1, 4}, {1, 2, 5}, {2, 3, 6}, {3, 0, 7}};
constexpr int H27_FACE[6][9] = {{0, 1, 2, 3, 8, 9, 10, 11, 20},  {0, 1, 5, 4, 8, 13, 16, 12, 21},
                                {1, 2, 6, 5, 9, 14, 17, 13, 22}, {2, 3, 7, 6, 10, 15, 18, 14, 23},
                                {3, 0, 4, 7, 11, 12, 19, 15, 24}, {4, 5, 6, 7, 16, 17, 18, 19, 25}};
// neighbour offset / outward normal of each side
constexpr int Q9_SIDE_DIR[4][3] = {{0, -1, 0}, {1, 0, 0}, {0, 1, 0}, {-1, 0, 0}};
constexpr int H27_FACE_DIR[6][3] = {{0, 0, -1}, {0, -1, 0}, {1, 0, 0}, {0, 1, 0}, {-1, 0, 0}, {0, 0, 1}};

}  // namespace exf
