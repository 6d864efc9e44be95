// Device-side views shared by the SW2 kernels and the host driver.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace sw2 {

// Static mesh data, laid out for coalesced per-element loads: every per-vertex
// field of a triangle is stored as three planes of length ntri (vertex a of
// element e at field[a*ntri + e]).  Segments follow the same scheme with two
// planes.  Elements are numbered triangles first, then segments
// (E = ntri + s), which is also the reference's assembly order
// (src/residual/assemble_residual.c:83-91, src/jacobian/assemble_jacobian.c:68-100).
struct MeshView {
    int nnodes, ntri, nseg;
    const int* tri;       // [ntri*3] node ids
    const double* ex;     // [3][ntri] vertex x
    const double* ey;     // [3][ntri] vertex y
    const double* ez;     // [3][ntri] bed elevation
    const double* gx;     // [3][ntri] d phi_a / dx
    const double* gy;     // [3][ntri] d phi_a / dy
    const double* djac;   // [ntri] area
    const int* seg;       // [nseg*2] node ids
    const double* snx;    // [nseg] outward normal
    const double* sny;
    const double* sdjac;  // [nseg] length
    const int* skind;     // [nseg] 0 velocity, 1 depth, 2 discharge, 3 tailwater, 4 outflow, 5 flux
    const double* sz0;    // [nseg] bed elevation of the segment's first node
};

struct StepParams {
    double dt;            // ts->dt / nsubsteps
    double alpha;         // tau_temporal
    double grav;
    double bc_depth, bc_vx, bc_vy;   // step-averaged series 0, 1, 2
    double bc_qs, bc_convey, bc_rough, bc_tail;   // discharge series value, conveyance, roughness height, tailwater elevation
    double bc_flux;                               // flux string's series value
};

// Deterministic assembly maps (built once from the bit-exact CSR):
//  residual: node n sums the entries ER[9*E + 3*a + v] listed in
//            rmap[rptr[n] .. rptr[n+1]) as E*3+a, in element order;
//  Jacobian: node-pair block k (CSR rows 3*i..3*i+2, columns 3*j..3*j+2) sums the
//            element blocks listed in jmap[jptr[k] .. jptr[k+1]) as E*9 + 3*a + b,
//            in element order, and writes vals[boff[k] + v*blen[k] + w].
struct AssemblyMaps {
    int nblocks;
    const int* rptr;      // [nnodes+1]
    const uint32_t* rmap;
    const int* jptr;      // [nblocks+1]
    const uint32_t* jmap;
    const int* boff;      // [nblocks] CSR position of (row 3i, column 3j)
    const int* blen;      // [nblocks] CSR row length of node i's rows
};

}  // namespace sw2
