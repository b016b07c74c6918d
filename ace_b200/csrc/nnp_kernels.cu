// nnp_kernels.cu -- the energy/force path on sm_100a.
//
// Stages (one launch each, all on the handle's stream):
//   k_atom_struct  atom -> structure map (binary search of the CSR offsets)
//   k_struct_setup per-structure cell grid in lattice coordinates
//   k_cell_base    exclusive scan of cells per structure
//   k_bin          wrap atoms into their cell, count atoms per cell
//   k_cell_start   per-structure scan of the cell counts
//   k_fill, k_sort_cells   cell member lists, sorted by type and atom index;
//                  the neighbour search's work items (a cell or a part of it)
//   k_prologue_small  the steps above in one thread block, for a periodic
//                  batch of at most 2048 atoms and 32 structures
//   k_neigh        one block per cell or part of a cell: candidates from the
//                  (2m+1)^3 cells gathered in shared memory, one warp per atom,
//                  exact FP64 displacement test, neighbours grouped by type
//                  (replaces NeighborList::build, struc/neighbor.cpp:46-87)
//   k_symm         one warp per atom: radial + angular symmetry functions
//                  (NNP::compute_symm, nnp/nnp.cpp:350-392)
//   k_nn_fp32      one warp per atom: network forward + input gradient dE/dG
//                  (ANN::fpbp + DODZ::grad, ml/nn.cpp:1402-1420,1836-1859)
//   k_force        one warp per atom: adjoint of the symmetry functions,
//                  per-neighbour gradients, FP64 force scatter
//                  (NNP::compute_force, nnp/nnp.cpp:412-476)
//   k_energy       one block per structure, FP64 energy sum
#include <cstdio>
#include <mutex>

#include "../../include/nnp_b200.h"
#include "nnp_device.cuh"
#include "nnp_engine.h"

namespace nnp {

#define FULL NNP_FULL
#define WARPS NNP_WARPS

__device__ __forceinline__ int floor_div(int a, int b) { return (a >= 0) ? a / b : -((-a + b - 1) / b); }

static int grid_for(int64_t items, int per_block, int max_blocks)
{
    int64_t b = (items + per_block - 1) / per_block;
    if (b < 1) b = 1;
    if (b > max_blocks) b = max_blocks;
    return (int)b;
}

static std::string cuda_msg(const char *what)
{
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) return "";
    return std::string(what) + ": " + cudaGetErrorString(e);
}

// ------------------------------------------------------------------ structure grids

__device__ __forceinline__ void atom_struct_one(int64_t i, const int64_t *__restrict__ off, int S,
                                                int *__restrict__ atom_struct, const int *__restrict__ type,
                                                int ntypes, DevErr *err)
{
    int lo = 0, hi = S - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (off[mid] <= i) lo = mid;
        else hi = mid - 1;
    }
    atom_struct[i] = lo;
    const int t = type[i];
    if (t < 0 || t >= ntypes) atomicMax(&err->bad_type, 1);
}

__global__ void k_atom_struct(const int64_t *__restrict__ off, int S, int64_t N, int *__restrict__ atom_struct,
                              const int *__restrict__ type, int ntypes, DevErr *err)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < N) atom_struct_one(i, off, S, atom_struct, type, ntypes, err);
}

// Atoms grouped by element: per-block counts in shared memory, one global
// atomic per (block, element) to count, then one to reserve each block's range.
// Atoms whose type is outside [0, ntypes) go last, in slot ntypes (the kernels
// that walk the order skip them; the call reports the bad type).
// Atoms [n_centre, N) are ghosts (neighbours only, never centres): they are
// counted with the out-of-range types, so `order` lists them last.
__global__ void k_type_count(int64_t N, int64_t n_centre, const int *__restrict__ type, int ntypes,
                             int *__restrict__ cnt)
{
    __shared__ int c[NNP_MAX_TYPES + 1];
    if (threadIdx.x <= NNP_MAX_TYPES) c[threadIdx.x] = 0;
    __syncthreads();
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < N) {
        const int t = type[i];
        atomicAdd(&c[(t >= 0 && t < ntypes && i < n_centre) ? t : ntypes], 1);
    }
    __syncthreads();
    if (threadIdx.x <= ntypes && c[threadIdx.x]) atomicAdd(&cnt[threadIdx.x], c[threadIdx.x]);
}

__global__ void k_type_scatter(int64_t N, int64_t n_centre, const int *__restrict__ type, int ntypes,
                               const int *__restrict__ cnt, int *__restrict__ fill, int *__restrict__ order)
{
    __shared__ int c[NNP_MAX_TYPES + 1], base[NNP_MAX_TYPES + 1];
    if (threadIdx.x <= NNP_MAX_TYPES) c[threadIdx.x] = 0;
    __syncthreads();
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int t = -1, r = 0;
    if (i < N) {
        t = type[i];
        if (!(t >= 0 && t < ntypes) || i >= n_centre) t = ntypes;
        r = atomicAdd(&c[t], 1);
    }
    __syncthreads();
    if (threadIdx.x <= ntypes) {
        int start = 0;
        for (int k = 0; k < (int)threadIdx.x; ++k) start += cnt[k];
        base[threadIdx.x] = start + (c[threadIdx.x] ? atomicAdd(&fill[threadIdx.x], c[threadIdx.x]) : 0);
    }
    __syncthreads();
    if (t >= 0) order[base[t] + r] = (int)i;
}

// Bounding box of every structure (free boundaries only): bbox[6s..6s+2] the
// smallest, bbox[6s+3..6s+5] the largest coordinate.  One block per structure.
__global__ void k_struct_bbox(const double *__restrict__ pos, const int64_t *__restrict__ off,
                              double *__restrict__ bbox)
{
    __shared__ double lo[3][256], hi[3][256];
    const int s = blockIdx.x, t = threadIdx.x;
    double l[3] = {1e300, 1e300, 1e300}, h[3] = {-1e300, -1e300, -1e300};
    for (int64_t a = off[s] + t; a < off[s + 1]; a += blockDim.x)
        for (int d = 0; d < 3; ++d) {
            const double x = pos[3 * a + d];
            l[d] = fmin(l[d], x);
            h[d] = fmax(h[d], x);
        }
    for (int d = 0; d < 3; ++d) { lo[d][t] = l[d]; hi[d][t] = h[d]; }
    __syncthreads();
    for (int k = blockDim.x / 2; k; k >>= 1) {
        if (t < k)
            for (int d = 0; d < 3; ++d) {
                lo[d][t] = fmin(lo[d][t], lo[d][t + k]);
                hi[d][t] = fmax(hi[d][t], hi[d][t + k]);
            }
        __syncthreads();
    }
    if (t == 0)
        for (int d = 0; d < 3; ++d) { bbox[6 * s + d] = lo[d][0]; bbox[6 * s + 3 + d] = hi[d][0]; }
}

// A free structure of more than this many atoms is searched through a cell
// grid over its bounding box (smaller ones are one cell, every atom a
// candidate of every other).
#define NNP_FREE_ONE_CELL 2048

__device__ void struct_setup_one(int s, const double *__restrict__ cell, const int64_t *__restrict__ off, int pbc,
                                 double rc, const double *__restrict__ bbox, StructGrid *__restrict__ grid,
                                 int *__restrict__ ncells, DevErr *err)
{
    StructGrid g;
    const int64_t nat = off[s + 1] - off[s];
    for (int k = 0; k < 9; ++k) { g.R[k] = 0.0; g.B[k] = 0.0; }
    g.nc[0] = g.nc[1] = g.nc[2] = 1;
    g.m[0] = g.m[1] = g.m[2] = 0;
    g.pbc = pbc;
    g.cell_base = 0;
    // A large free structure is put in an orthorhombic periodic box at least
    // rc (+1 A) wider than its bounding box in every direction, so no periodic
    // image of an atom comes within rc of another: the cell-list search of the
    // periodic path then finds exactly the free structure's neighbours.
    const bool boxed = !pbc && nat > NNP_FREE_ONE_CELL;
    if (boxed) {
        for (int d = 0; d < 3; ++d) g.R[4 * d] = (bbox[6 * s + 3 + d] - bbox[6 * s + d]) + rc + 1.0;
        g.pbc = 1;
    }
    if (pbc || boxed) {
        if (pbc)
            for (int k = 0; k < 9; ++k) g.R[k] = cell[9 * (int64_t)s + k];
        const double *a[3] = {g.R, g.R + 3, g.R + 6};
        double c[3][3];
        for (int n = 0; n < 3; ++n) {
            const double *p = a[(n + 1) % 3], *q = a[(n + 2) % 3];
            c[n][0] = p[1] * q[2] - p[2] * q[1];
            c[n][1] = p[2] * q[0] - p[0] * q[2];
            c[n][2] = p[0] * q[1] - p[1] * q[0];
        }
        const double V = a[0][0] * c[0][0] + a[0][1] * c[0][1] + a[0][2] * c[0][2];
        if (!(fabs(V) > 1e-12)) {
            atomicMax(&err->bad_cell, 1);
            g.pbc = 0;
        } else {
            double w[3];
            for (int n = 0; n < 3; ++n) {
                for (int d = 0; d < 3; ++d) g.B[3 * n + d] = c[n][d] / V;
                w[n] = fabs(V) / sqrt(c[n][0] * c[n][0] + c[n][1] * c[n][1] + c[n][2] * c[n][2]);
                int nc = (int)floor(w[n] / rc);
                g.nc[n] = nc < 1 ? 1 : (nc > 1024 ? 1024 : nc);
            }
            const int64_t lim = nat * 2 > 64 ? nat * 2 : 64;
            while ((int64_t)g.nc[0] * g.nc[1] * g.nc[2] > lim) {
                int k = 0;
                if (g.nc[1] > g.nc[k]) k = 1;
                if (g.nc[2] > g.nc[k]) k = 2;
                g.nc[k] = (g.nc[k] + 1) / 2;
            }
            for (int n = 0; n < 3; ++n) g.m[n] = (int)fmin(ceil(rc * g.nc[n] / w[n]), 1e6);
            if (g.m[0] > NNP_MAX_IMAGES || g.m[1] > NNP_MAX_IMAGES || g.m[2] > NNP_MAX_IMAGES) {
                // thinner than rc / NNP_MAX_IMAGES in some direction: reported, not searched
                atomicMax(&err->bad_cell, 2);
                g.m[0] = g.m[1] = g.m[2] = 0;
            }
        }
    }
    grid[s] = g;
    ncells[s] = g.nc[0] * g.nc[1] * g.nc[2];
}

__global__ void k_struct_setup(const double *__restrict__ cell, const int64_t *__restrict__ off, int S, int pbc,
                               double rc, const double *__restrict__ bbox, StructGrid *__restrict__ grid,
                               int *__restrict__ ncells, DevErr *err)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < S) struct_setup_one(s, cell, off, pbc, rc, bbox, grid, ncells, err);
}

// exclusive scan of ncells over structures in one block; writes cell_base
__global__ void k_cell_base(const int *__restrict__ ncells, int S, StructGrid *__restrict__ grid)
{
    __shared__ int part[1024];
    const int t = threadIdx.x, T = blockDim.x;
    const int chunk = (S + T - 1) / T;
    const int b = t * chunk, e = min(S, b + chunk);
    int s = 0;
    for (int k = b; k < e; ++k) s += ncells[k];
    part[t] = s;
    __syncthreads();
    for (int d = 1; d < T; d <<= 1) {
        const int v = (t >= d) ? part[t - d] : 0;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    int run = part[t] - s;
    for (int k = b; k < e; ++k) {
        grid[k].cell_base = run;
        run += ncells[k];
    }
}

__device__ __forceinline__ void bin_one(int64_t i, const double *__restrict__ pos, const int *__restrict__ atom_struct,
                                        const StructGrid *__restrict__ grid, double *__restrict__ xw,
                                        int *__restrict__ atom_cell, int *__restrict__ cell_cnt)
{
    const StructGrid &g = grid[atom_struct[i]];
    const double x[3] = {pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
    int cid = g.cell_base;
    double y[3] = {x[0], x[1], x[2]};
    if (g.pbc) {
        int c[3];
        double sh[3];
        for (int n = 0; n < 3; ++n) {
            const double f = g.B[3 * n] * x[0] + g.B[3 * n + 1] * x[1] + g.B[3 * n + 2] * x[2];
            double k = floor(f);
            double fw = f - k;
            if (fw >= 1.0) { fw -= 1.0; k += 1.0; }
            if (fw < 0.0) fw = 0.0;
            sh[n] = k;
            int cc = (int)(fw * g.nc[n]);
            c[n] = cc >= g.nc[n] ? g.nc[n] - 1 : cc;
        }
        for (int d = 0; d < 3; ++d) y[d] = x[d] - (g.R[d] * sh[0] + g.R[3 + d] * sh[1] + g.R[6 + d] * sh[2]);
        cid += (c[0] * g.nc[1] + c[1]) * g.nc[2] + c[2];
    }
    xw[3 * i] = y[0];
    xw[3 * i + 1] = y[1];
    xw[3 * i + 2] = y[2];
    atom_cell[i] = cid;
    atomicAdd(&cell_cnt[cid], 1);
}

__global__ void k_bin(int64_t N, const double *__restrict__ pos, const int *__restrict__ atom_struct,
                      const StructGrid *__restrict__ grid, double *__restrict__ xw, int *__restrict__ atom_cell,
                      int *__restrict__ cell_cnt)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < N) bin_one(i, pos, atom_struct, grid, xw, atom_cell, cell_cnt);
}

// one block per structure: exclusive scan of its cells' counts
__global__ void k_cell_start(const StructGrid *__restrict__ grid, const int *__restrict__ ncells,
                             const int *__restrict__ cell_cnt, int *__restrict__ cell_start, int *__restrict__ cell_fill,
                             const int64_t *__restrict__ off)
{
    __shared__ int part[256];
    const int s = blockIdx.x, t = threadIdx.x, T = blockDim.x;
    const int base = grid[s].cell_base, nc = ncells[s];
    const int chunk = (nc + T - 1) / T;
    const int b = t * chunk, e = min(nc, b + chunk);
    int sum = 0;
    for (int k = b; k < e; ++k) sum += cell_cnt[base + k];
    part[t] = sum;
    __syncthreads();
    for (int d = 1; d < T; d <<= 1) {
        const int v = (t >= d) ? part[t - d] : 0;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    int run = (int)off[s] + part[t] - sum;
    for (int k = b; k < e; ++k) {
        cell_start[base + k] = run;
        cell_fill[base + k] = 0;
        run += cell_cnt[base + k];
    }
}

__global__ void k_fill(int64_t N, const int *__restrict__ atom_cell, const int *__restrict__ cell_start,
                       int *__restrict__ cell_fill, int *__restrict__ cell_atoms)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= N) return;
    const int c = atom_cell[i];
    const int slot = cell_start[c] + atomicAdd(&cell_fill[c], 1);
    cell_atoms[slot] = (int)i;
}

#define NEIGH_WARPS 4         // warps per block of the neighbour search
#define NEIGH_THREADS (NEIGH_WARPS * 32)
#define NEIGH_BLOCKS 7        // resident blocks per SM (shared memory)
#define NEIGH_CAND 768       // candidates held in shared memory at a time (multiple of 64)
#define NEIGH_ENT 512         // (type, neighbouring cell) segments of one cell's candidate list
#define NEIGH_ATOMS 1024      // atoms of one cell whose counts are kept while chunks stream
#define NEIGH_ITEM_COUNTER (2 * (NNP_MAX_TYPES + 1))   // type_fill entry counting the neighbour-search work items

// Work items of the neighbour search: the atoms of a cell split into parts of
// about `budget` candidate tests (atoms x candidates, the candidates estimated
// as the cell's own count times the O = (2m+1)^3 cells searched), one atom
// per warp at the finest.  A big cell (a small periodic structure is one cell
// seen through its 27 images) then spreads over several blocks instead of
// setting the search's time on one.
__device__ __forceinline__ int neigh_parts(int n, int O, int budget)
{
    if (n <= 0) return 0;
    const int64_t p = ((int64_t)O * n * n + budget - 1) / budget;
    const int pmax = (n + NEIGH_WARPS - 1) / NEIGH_WARPS;
    return (int)(p < 1 ? 1 : (p > pmax ? pmax : p));
}

// Sort key of a cell member: type in the top 4 bits (atom indices < 2^28); a
// type outside [0, ntypes) gets 15, sorts last and is counted for no type.
__device__ __forceinline__ unsigned sort_key(int atom, int t, int ntypes)
{
    const unsigned tt = (t >= 0 && t < ntypes) ? (unsigned)t : 15u;
    return (unsigned)atom | (tt << 28);
}

// The members of every cell (all structures) sorted by (type, atom index)
// and counted per type, and the cell's neighbour-search work items; one warp
// per cell, the warps striding over all cells.  The keys type << 28 | atom
// are distinct, so a key's place is the number of smaller keys (the same
// order as any comparison sort): a cell of at most 32 atoms has one key per
// lane, a larger one is ranked four keys per lane per load of a compared key.
// The keys sit in the warp's shared memory, or for a cell of more than
// SORT_SMEM atoms (a free structure of up to NNP_FREE_ONE_CELL atoms is one
// cell) in tmp at the cell's own slots.  Each cell appends its parts
// (neigh_parts) to `items` as {cell, structure, first atom, end atom}, at a
// place taken from items_n.
#define SORT_WARPS 4
#define SORT_SMEM 512
// one cell by one warp; keys: the warp's shared buffer of kcap entries
__device__ void sort_cell(int c, int lane, unsigned *keys, int kcap, const StructGrid *__restrict__ grid,
                          const int *__restrict__ cell_cnt, const int *__restrict__ cell_start,
                          const int *__restrict__ type, const int *__restrict__ atom_struct, int ntypes, int budget,
                          int *__restrict__ cell_atoms, int *__restrict__ cell_tcnt, unsigned *__restrict__ tmp,
                          int4 *__restrict__ items, int *__restrict__ items_n)
{
    const int n = cell_cnt[c];
    if (n == 0) return;                                          // uniform over the warp
    const int cs = cell_start[c];
    int *a = cell_atoms + cs;
    unsigned *k = (n <= kcap) ? keys : tmp + cs;
    for (int p = lane; p < n; p += 32) k[p] = sort_key(a[p], type[a[p]], ntypes);
    int s = 0, parts = 0, base = 0;
    if (lane == 0) {
        s = atom_struct[a[0]];
        const StructGrid &g = grid[s];
        parts = neigh_parts(n, (2 * g.m[0] + 1) * (2 * g.m[1] + 1) * (2 * g.m[2] + 1), budget);
        base = atomicAdd(items_n, parts);
    }
    s = __shfl_sync(0xffffffffu, s, 0);
    parts = __shfl_sync(0xffffffffu, parts, 0);
    base = __shfl_sync(0xffffffffu, base, 0);
    for (int p = lane; p < parts; p += 32)
        items[base + p] = make_int4(c, s, (int)((int64_t)p * n / parts), (int)((int64_t)(p + 1) * n / parts));
    __threadfence_block();
    __syncwarp();                                                // keys written, a[0] read
    int *tc = cell_tcnt + (size_t)c * ntypes;
    if (n <= 32) {
        const unsigned v = lane < n ? k[lane] : 0xffffffffu;
        int r = 0;
        for (int q = 0; q < n; ++q) r += (k[q] < v) ? 1 : 0;
        if (lane < n) a[r] = (int)(v & 0x0fffffffu);
        for (int t = 0; t < ntypes; ++t) {
            const int m = __popc(__ballot_sync(0xffffffffu, lane < n && (v >> 28) == (unsigned)t));
            if (lane == 0) tc[t] = m;
        }
    } else {
        for (int p0 = lane; p0 < n; p0 += 128) {
            unsigned v[4];
            int r[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                v[u] = (p0 + 32 * u < n) ? k[p0 + 32 * u] : 0xffffffffu;
                r[u] = 0;
            }
            for (int q = 0; q < n; ++q) {
                const unsigned w = k[q];
#pragma unroll
                for (int u = 0; u < 4; ++u) r[u] += (w < v[u]) ? 1 : 0;
            }
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (p0 + 32 * u < n) a[r[u]] = (int)(v[u] & 0x0fffffffu);
        }
        for (int t = 0; t < ntypes; ++t) {
            int m = 0;
            for (int p = lane; p < n; p += 32) m += ((k[p] >> 28) == (unsigned)t) ? 1 : 0;
#pragma unroll
            for (int o = 16; o; o >>= 1) m += __shfl_xor_sync(0xffffffffu, m, o);
            if (lane == 0) tc[t] = m;
        }
    }
    __syncwarp();                                                // keys reused by the next cell
}

__global__ void __launch_bounds__(SORT_WARPS * 32)
k_sort_cells(int S, const StructGrid *__restrict__ grid, const int *__restrict__ ncells,
             const int *__restrict__ cell_cnt, const int *__restrict__ cell_start, const int *__restrict__ type,
             const int *__restrict__ atom_struct, int ntypes, int budget, int *__restrict__ cell_atoms,
             int *__restrict__ cell_tcnt, unsigned *__restrict__ tmp, int4 *__restrict__ items,
             int *__restrict__ items_n)
{
    __shared__ unsigned keys[SORT_WARPS][SORT_SMEM];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int total = grid[S - 1].cell_base + ncells[S - 1];
    for (int c = blockIdx.x * SORT_WARPS + warp; c < total; c += gridDim.x * SORT_WARPS)
        sort_cell(c, lane, keys[warp], SORT_SMEM, grid, cell_cnt, cell_start, type, atom_struct, ntypes, budget,
                  cell_atoms, cell_tcnt, tmp, items, items_n);
}

__device__ __forceinline__ void cell_pos_one(int64_t s, const int *__restrict__ cell_atoms,
                                             const double *__restrict__ xw, const int *__restrict__ type, int ntypes,
                                             double4 *__restrict__ cell_pos)
{
    const int a = cell_atoms[s];
    const int t = type[a];
    cell_pos[s] = make_double4(xw[3 * (int64_t)a], xw[3 * (int64_t)a + 1], xw[3 * (int64_t)a + 2],
                               (t >= 0 && t < ntypes) ? (double)t : -1.0);
}

__global__ void k_cell_pos(int64_t N, const int *__restrict__ cell_atoms, const double *__restrict__ xw,
                           const int *__restrict__ type, int ntypes, double4 *__restrict__ cell_pos)
{
    const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (s < N) cell_pos_one(s, cell_atoms, xw, type, ntypes, cell_pos);
}

// The neighbour-search prologue of a small periodic batch (one MD-style cell
// or a few) in one thread block: the steps of the launch sequence k_type_count
// ... k_cell_pos with block barriers between them instead of launches, on the
// same device functions.  Element counts and fill cursors land in type_fill
// as k_type_count / k_type_scatter leave them; `order` lists each element's
// atoms in some order (every consumer treats atoms independently); cell
// starts are one warp's scan per structure.
#define PRO_THREADS 1024
#define PRO_MAX_ATOMS 2048
#define PRO_MAX_STRUCT 32
#define PRO_SORT_SMEM 256
__global__ void __launch_bounds__(PRO_THREADS)
k_prologue_small(int64_t N, int64_t n_centre, int S, int cell_bound, const int64_t *__restrict__ off,
                 const double *__restrict__ pos, const double *__restrict__ cell, const int *__restrict__ type,
                 int ntypes, double rc, int budget, StructGrid *__restrict__ grid, int *__restrict__ ncells,
                 int *__restrict__ atom_struct, double *__restrict__ xw, int *__restrict__ atom_cell,
                 int *__restrict__ cell_cnt, int *__restrict__ cell_start, int *__restrict__ cell_fill,
                 int *__restrict__ cell_atoms, int *__restrict__ cell_tcnt, double4 *__restrict__ cell_pos,
                 int *__restrict__ type_fill, int *__restrict__ order, int4 *__restrict__ items, DevErr *err)
{
    __shared__ int cnt[NNP_MAX_TYPES + 1], cur[NNP_MAX_TYPES + 1], tbase[NNP_MAX_TYPES + 1];
    __shared__ unsigned keys[PRO_THREADS / 32][PRO_SORT_SMEM];
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    int *items_n = type_fill + NEIGH_ITEM_COUNTER;
    if (t <= NNP_MAX_TYPES) {
        cnt[t] = 0;
        cur[t] = 0;
    }
    if (t == 0) *items_n = 0;
    for (int c = t; c < cell_bound; c += PRO_THREADS) cell_cnt[c] = 0;
    __syncthreads();
    // atom -> structure, element counts (ghosts and bad types in slot ntypes), structure grids
    for (int64_t i = t; i < N; i += PRO_THREADS) {
        atom_struct_one(i, off, S, atom_struct, type, ntypes, err);
        const int ty = type[i];
        atomicAdd(&cnt[(ty >= 0 && ty < ntypes && i < n_centre) ? ty : ntypes], 1);
    }
    for (int s = t; s < S; s += PRO_THREADS) struct_setup_one(s, cell, off, 1, rc, nullptr, grid, ncells, err);
    __syncthreads();
    if (t <= NNP_MAX_TYPES) {
        int b = 0;
        for (int k = 0; k < t && k <= ntypes; ++k) b += cnt[k];
        tbase[t] = b;
        type_fill[t] = (t <= ntypes) ? cnt[t] : 0;
        type_fill[NNP_MAX_TYPES + 1 + t] = (t <= ntypes) ? cnt[t] : 0;
    }
    if (t == 0) {
        int run = 0;
        for (int s = 0; s < S; ++s) {
            grid[s].cell_base = run;
            run += ncells[s];
        }
    }
    __syncthreads();
    // visiting order by element; wrapped positions, cell of each atom, counts
    for (int64_t i = t; i < N; i += PRO_THREADS) {
        int ty = type[i];
        if (!(ty >= 0 && ty < ntypes) || i >= n_centre) ty = ntypes;
        order[tbase[ty] + atomicAdd(&cur[ty], 1)] = (int)i;
        bin_one(i, pos, atom_struct, grid, xw, atom_cell, cell_cnt);
    }
    __syncthreads();
    for (int s = warp; s < S; s += PRO_THREADS / 32) {
        const int base = grid[s].cell_base, nc = ncells[s];
        int run = (int)off[s];
        for (int c0 = 0; c0 < nc; c0 += 32) {
            const int c = c0 + lane;
            const int v = c < nc ? cell_cnt[base + c] : 0;
            int inc = v;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const int u = __shfl_up_sync(0xffffffffu, inc, d);
                if (lane >= d) inc += u;
            }
            if (c < nc) {
                cell_start[base + c] = run + inc - v;
                cell_fill[base + c] = 0;
            }
            run += __shfl_sync(0xffffffffu, inc, 31);
        }
    }
    __syncthreads();
    for (int64_t i = t; i < N; i += PRO_THREADS) {
        const int c = atom_cell[i];
        cell_atoms[cell_start[c] + atomicAdd(&cell_fill[c], 1)] = (int)i;
    }
    __syncthreads();
    // (atom_cell, read above, holds the keys of cells larger than the shared buffer)
    const int total = grid[S - 1].cell_base + ncells[S - 1];
    for (int c = warp; c < total; c += PRO_THREADS / 32)
        sort_cell(c, lane, keys[warp], PRO_SORT_SMEM, grid, cell_cnt, cell_start, type, atom_struct, ntypes, budget,
                  cell_atoms, cell_tcnt, reinterpret_cast<unsigned *>(atom_cell), items, items_n);
    __syncthreads();
    for (int64_t k = t; k < N; k += PRO_THREADS) cell_pos_one(k, cell_atoms, xw, type, ntypes, cell_pos);
}

// Neighbour search, one thread block per work item: a cell, or a part of its
// atoms (k_sort_cells).  Every atom of a cell has the same candidates: the members of the (2m+1)^3 cells around it, each with its
// lattice image shift.  The block gathers them into shared memory with the
// shift applied in FP64 (x_j + R q), ordered by neighbour type, then by cell
// offset, then by atom index (cell member lists are sorted by type and index),
// and each warp tests one atom of the cell against the list: the FP64
// displacement x_i - (x_j + R q) decides membership (r^2 < rc^2; a self image
// needs r^2 > 1e-12 as in neighbor.cpp:78).  Accepted candidates are written
// in list order, so each atom's list comes out grouped by type:
// float4(dx,dy,dz, j | type<<28).  Candidate lists longer than the shared
// buffer stream through it in chunks; a cell with more (type, cell) segments
// than the segment table holds is searched from global memory, one warp per
// atom, with the same order and arithmetic.

struct NeighShared {
    union {
        struct {
            double x[NEIGH_CAND], y[NEIGH_CAND], z[NEIGH_CAND];   // shifted candidate positions
            int jt[NEIGH_CAND];                                  // j | type << 28
        } c;
        float4 lst[NEIGH_WARPS][NNP_MAX_NBR]; // global-memory search: accepted, j | type << 28 in .w
    };
    int count[NEIGH_ATOMS];                   // running neighbour counts (chunked lists)
    int pre[NEIGH_ENT + 1];                   // exclusive scan of the segment lengths
    int start[NEIGH_ENT];                     // first member slot of each segment
    int q[NEIGH_ENT];                         // image shift of each segment, 3 x 8 bits
};

__device__ __forceinline__ int pack_q(int q0, int q1, int q2)
{
    return (q0 + 128) | ((q1 + 128) << 8) | ((q2 + 128) << 16);
}

// neighbouring cell o of local cell (c0,c1,c2): global index and image shift
__device__ __forceinline__ int cell_offset(const StructGrid &g, int c0, int c1, int c2, int o, int &q0, int &q1, int &q2)
{
    const int w1 = 2 * g.m[1] + 1, w2 = 2 * g.m[2] + 1;
    const int d2 = o % w2 - g.m[2];
    const int t = o / w2;
    const int d1 = t % w1 - g.m[1];
    const int d0 = t / w1 - g.m[0];
    const int t0 = c0 + d0, t1 = c1 + d1, t2 = c2 + d2;
    q0 = floor_div(t0, g.nc[0]);
    q1 = floor_div(t1, g.nc[1]);
    q2 = floor_div(t2, g.nc[2]);
    return g.cell_base + ((t0 - q0 * g.nc[0]) * g.nc[1] + (t1 - q1 * g.nc[1])) * g.nc[2] + (t2 - q2 * g.nc[2]);
}

// Candidates [k0, k1) of the cell's list into shared memory slots [0, k1-k0),
// slots up to kp filled with NaN positions (never accepted).
__device__ __forceinline__ void load_candidates(NeighShared &sh, int k0, int k1, int kp, int NE, const StructGrid &g,
                                                const double4 *__restrict__ cell_pos,
                                                const int *__restrict__ cell_atoms, int tid)
{
    const double R0 = g.R[0], R1 = g.R[1], R2 = g.R[2], R3 = g.R[3], R4 = g.R[4], R5 = g.R[5], R6 = g.R[6],
                 R7 = g.R[7], R8 = g.R[8];
    for (int s = tid; s < kp; s += NEIGH_THREADS) {
        const int k = k0 + s;
        if (k >= k1) {
            const double nan = __longlong_as_double(0x7ff8000000000000ll);
            sh.c.x[s] = sh.c.y[s] = sh.c.z[s] = nan;
            sh.c.jt[s] = 0;
            continue;
        }
        int lo = 0, hi = NE;                                     // last segment with pre <= k
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (sh.pre[mid] <= k) lo = mid; else hi = mid;
        }
        const int slot = sh.start[lo] + k - sh.pre[lo];
        const double4 xj = cell_pos[slot];
        const int j = cell_atoms[slot];
        if (xj.w < 0.0) {                                        // type out of range: never a neighbour
            const double nan = __longlong_as_double(0x7ff8000000000000ll);
            sh.c.x[s] = sh.c.y[s] = sh.c.z[s] = nan;
            sh.c.jt[s] = 0;
            continue;
        }
        const int qp = sh.q[lo];
        const double Q0 = (qp & 255) - 128, Q1 = ((qp >> 8) & 255) - 128, Q2 = ((qp >> 16) & 255) - 128;
        sh.c.x[s] = xj.x + (R0 * Q0 + R3 * Q1 + R6 * Q2);
        sh.c.y[s] = xj.y + (R1 * Q0 + R4 * Q1 + R7 * Q2);
        sh.c.z[s] = xj.z + (R2 * Q0 + R5 * Q1 + R8 * Q2);
        sh.c.jt[s] = j | ((int)xj.w << 28);
    }
}

// Tests atom i against shared slots [0, kp) (kp a multiple of 64, two batches
// of 32 in flight), appending accepted candidates to out[count..cap) in slot
// order; returns the new count.
__device__ __forceinline__ int test_candidates(const NeighShared &sh, int kp, int lane, int i, double xi0, double xi1,
                                               double xi2, double rc2, int count, int cap, float4 *__restrict__ out)
{
    const unsigned lt = (1u << lane) - 1u;
    for (int kb = 0; kb < kp; kb += 64) {
        const int ka = kb + lane, kc = ka + 32;
        const double ax = xi0 - sh.c.x[ka], ay = xi1 - sh.c.y[ka], az = xi2 - sh.c.z[ka];
        const double cx = xi0 - sh.c.x[kc], cy = xi1 - sh.c.y[kc], cz = xi2 - sh.c.z[kc];
        const double ra = ax * ax + ay * ay + az * az, rb = cx * cx + cy * cy + cz * cz;
        bool acca = ra < rc2, accb = rb < rc2;
        if (acca && !(ra > 1e-12)) acca = (sh.c.jt[ka] & 0x0fffffff) != i;
        if (accb && !(rb > 1e-12)) accb = (sh.c.jt[kc] & 0x0fffffff) != i;
        const unsigned ba = __ballot_sync(FULL, acca), bb = __ballot_sync(FULL, accb);
        if (acca) {
            const int p = count + __popc(ba & lt);
            if (p < cap) out[p] = make_float4((float)ax, (float)ay, (float)az, __int_as_float(sh.c.jt[ka]));
        }
        count += __popc(ba);
        if (accb) {
            const int p = count + __popc(bb & lt);
            if (p < cap) out[p] = make_float4((float)cx, (float)cy, (float)cz, __int_as_float(sh.c.jt[kc]));
        }
        count += __popc(bb);
    }
    return count;
}

__device__ __forceinline__ void finish_atom(int64_t i, int count, int cap, int *__restrict__ nbr_cnt, DevErr *err)
{
    nbr_cnt[i] = min(count, cap);
    if (count > cap) atomicMax(&err->need_cap, count);
}

// Global-memory search of one atom: lanes take 32 neighbouring cells at a
// time and then their members, located by a binary search over the lanes'
// running counts; accepted neighbours are staged in candidate order and then
// written grouped by type.
__device__ void search_atom_global(NeighShared &sh, int warp, int lane, int64_t i, const StructGrid &g, int c0, int c1,
                                   int c2, double xi0, double xi1, double xi2, const double4 *__restrict__ cell_pos,
                                   const int *__restrict__ cell_cnt, const int *__restrict__ cell_start,
                                   const int *__restrict__ cell_atoms, double rc2, int cap, int ntypes,
                                   float4 *__restrict__ nbr, int *__restrict__ nbr_cnt, DevErr *err)
{
    const unsigned lt = (1u << lane) - 1u;
    const int O = (2 * g.m[0] + 1) * (2 * g.m[1] + 1) * (2 * g.m[2] + 1);
    int count = 0;
    for (int ob = 0; ob < O; ob += 32) {
        const int o = ob + lane;
        int cnt = 0, start = 0, q0 = 0, q1 = 0, q2 = 0;
        if (o < O) {
            const int cw = cell_offset(g, c0, c1, c2, o, q0, q1, q2);
            cnt = cell_cnt[cw];
            start = cell_start[cw];
        }
        int inc = cnt;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int v = __shfl_up_sync(FULL, inc, d);
            if (lane >= d) inc += v;
        }
        const int exc = inc - cnt;
        const int total = __shfl_sync(FULL, inc, 31);
        for (int kb = 0; kb < total; kb += 32) {
            const int k = kb + lane;
            int lo = 0;
#pragma unroll
            for (int step = 16; step; step >>= 1) {
                const int ex = __shfl_sync(FULL, exc, lo + step);
                if (ex <= k) lo += step;
            }
            const int st = __shfl_sync(FULL, start, lo);
            const int ex = __shfl_sync(FULL, exc, lo);
            const double Q0 = __shfl_sync(FULL, q0, lo), Q1 = __shfl_sync(FULL, q1, lo), Q2 = __shfl_sync(FULL, q2, lo);
            bool acc = false;
            float4 e = make_float4(0.f, 0.f, 0.f, 0.f);
            if (k < total) {
                const int slot = st + k - ex;
                const int j = cell_atoms[slot];
                const double4 xj = cell_pos[slot];
                const double dx = xi0 - (xj.x + (g.R[0] * Q0 + g.R[3] * Q1 + g.R[6] * Q2));
                const double dy = xi1 - (xj.y + (g.R[1] * Q0 + g.R[4] * Q1 + g.R[7] * Q2));
                const double dz = xi2 - (xj.z + (g.R[2] * Q0 + g.R[5] * Q1 + g.R[8] * Q2));
                const double r2 = dx * dx + dy * dy + dz * dz;
                if (r2 < rc2 && ((int64_t)j != i || r2 > 1e-12) && xj.w >= 0.0) {
                    acc = true;
                    e = make_float4((float)dx, (float)dy, (float)dz, __int_as_float(j | ((int)xj.w << 28)));
                }
            }
            const unsigned bal = __ballot_sync(FULL, acc);
            const int p = count + __popc(bal & lt);
            if (acc && p < NNP_MAX_NBR) sh.lst[warp][p] = e;
            count += __popc(bal);
        }
    }
    __syncwarp();
    const int nw = min(count, NNP_MAX_NBR);
    int outp = 0;
    for (int t = 0; t < ntypes; ++t) {
        for (int kb = 0; kb < nw; kb += 32) {
            const int k = kb + lane;
            float4 e = make_float4(0.f, 0.f, 0.f, 0.f);
            bool m = false;
            if (k < nw) {
                e = sh.lst[warp][k];
                m = ((unsigned)__float_as_int(e.w) >> 28) == (unsigned)t;
            }
            const unsigned bal = __ballot_sync(FULL, m);
            const int p = outp + __popc(bal & lt);
            if (m && p < cap) nbr[i * cap + p] = e;
            outp += __popc(bal);
        }
    }
    if (lane == 0) finish_atom(i, count, cap, nbr_cnt, err);
    __syncwarp();
}

__global__ void __launch_bounds__(NEIGH_THREADS, NEIGH_BLOCKS) k_neigh(const int4 *__restrict__ items,
                                                          const int *__restrict__ items_n,
                                                          const StructGrid *__restrict__ grid,
                                                          const double4 *__restrict__ cell_pos,
                                                          const int *__restrict__ cell_cnt,
                                                          const int *__restrict__ cell_start,
                                                          const int *__restrict__ cell_tcnt,
                                                          const int *__restrict__ cell_atoms, double rc2, int cap,
                                                          int ntypes, float4 *__restrict__ nbr,
                                                          int *__restrict__ nbr_cnt, DevErr *err)
{
    extern __shared__ __align__(16) unsigned char neigh_smem[];
    NeighShared &sh = *reinterpret_cast<NeighShared *>(neigh_smem);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int nitems = *items_n;
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {  // uniform over the block
        const int4 w = items[it];
        const int c = w.x, a_lo = w.z, a_hi = w.w;
        const int cs = cell_start[c];
        const StructGrid &g = grid[w.y];
        const int local = c - g.cell_base;
        const int c2 = local % g.nc[2], c1 = (local / g.nc[2]) % g.nc[1], c0 = local / (g.nc[1] * g.nc[2]);
        const int O = (2 * g.m[0] + 1) * (2 * g.m[1] + 1) * (2 * g.m[2] + 1);
        const int NE = ntypes * O;
        if (NE > NEIGH_ENT) {
            for (int a = a_lo + warp; a < a_hi; a += NEIGH_WARPS) {
                const double4 xi = cell_pos[cs + a];
                search_atom_global(sh, warp, lane, cell_atoms[cs + a], g, c0, c1, c2, xi.x, xi.y, xi.z, cell_pos,
                                   cell_cnt, cell_start, cell_atoms, rc2, cap, ntypes, nbr, nbr_cnt, err);
            }
            __syncthreads();
            continue;
        }
        // segments (type t, neighbouring cell o), type-major
        for (int e = tid; e < NE; e += NEIGH_THREADS) {
            const int t = e / O, o = e - t * O;
            int q0, q1, q2;
            const int cw = cell_offset(g, c0, c1, c2, o, q0, q1, q2);
            const int *tc = cell_tcnt + (size_t)cw * ntypes;
            int s0 = cell_start[cw];
            for (int u = 0; u < t; ++u) s0 += tc[u];
            sh.pre[e + 1] = tc[t];
            sh.start[e] = s0;
            sh.q[e] = pack_q(q0, q1, q2);
        }
        __syncthreads();
        if (warp == 0) {
            int run = 0;
            for (int eb = 0; eb < NE; eb += 32) {
                const int e = eb + lane;
                const int v = e < NE ? sh.pre[e + 1] : 0;
                int inc = v;
#pragma unroll
                for (int d = 1; d < 32; d <<= 1) {
                    const int u = __shfl_up_sync(FULL, inc, d);
                    if (lane >= d) inc += u;
                }
                if (e < NE) sh.pre[e + 1] = run + inc;
                run += __shfl_sync(FULL, inc, 31);
            }
            if (lane == 0) sh.pre[0] = 0;
        }
        __syncthreads();
        const int T = sh.pre[NE];
        if (T <= NEIGH_CAND) {
            const int kp = (T + 63) & ~63;
            load_candidates(sh, 0, T, kp, NE, g, cell_pos, cell_atoms, tid);
            __syncthreads();
            for (int a = a_lo + warp; a < a_hi; a += NEIGH_WARPS) {
                const int i = cell_atoms[cs + a];
                const double4 xi = cell_pos[cs + a];
                const int count = test_candidates(sh, kp, lane, i, xi.x, xi.y, xi.z, rc2, 0, cap, nbr + (int64_t)i * cap);
                if (lane == 0) finish_atom(i, count, cap, nbr_cnt, err);
            }
        } else {
            for (int a0 = a_lo; a0 < a_hi; a0 += NEIGH_ATOMS) {
                const int a1 = min(a_hi, a0 + NEIGH_ATOMS);
                for (int a = a0 + tid; a < a1; a += NEIGH_THREADS) sh.count[a - a0] = 0;
                for (int k0 = 0; k0 < T; k0 += NEIGH_CAND) {
                    const int k1 = min(T, k0 + NEIGH_CAND), kp = (k1 - k0 + 63) & ~63;
                    __syncthreads();                             // the previous chunk is tested
                    load_candidates(sh, k0, k1, kp, NE, g, cell_pos, cell_atoms, tid);
                    __syncthreads();
                    for (int a = a0 + warp; a < a1; a += NEIGH_WARPS) {
                        const int i = cell_atoms[cs + a];
                        const double4 xi = cell_pos[cs + a];
                        const int count = test_candidates(sh, kp, lane, i, xi.x, xi.y, xi.z, rc2, sh.count[a - a0],
                                                          cap, nbr + (int64_t)i * cap);
                        __syncwarp();
                        if (lane == 0) sh.count[a - a0] = count;
                    }
                }
                __syncthreads();
                for (int a = a0 + tid; a < a1; a += NEIGH_THREADS) finish_atom(cell_atoms[cs + a], sh.count[a - a0], cap, nbr_cnt, err);
            }
        }
        __syncthreads();                                         // the shared lists are reused by the next cell
    }
}

// ------------------------------------------------------------------ symmetry functions

// Acc is the type of the per-lane running sums: each lane adds up to T/32 pair
// terms of one function, so FP32 sums lose ~sqrt(T/32) ulps; FP64 sums keep G
// to the FP32 rounding of the final value.
template <typename Acc>
__global__ void __launch_bounds__(WARPS * 32, 1) k_symm(int64_t N, const DevPot *__restrict__ pot,
                                                       const float2 *__restrict__ rpar, const float4 *__restrict__ apar,
                                                       const int *__restrict__ type, const int *__restrict__ order, const float4 *__restrict__ nbr,
                                                       const int *__restrict__ nbr_cnt, int cap, int ncut_max, int ndamp_max,
                                                       int gstride, float *__restrict__ G)
{
    extern __shared__ float4 smem4[];
    symm_body<Acc, GenericBlocks>(N, pot, rpar, apar, type, order, nbr, nbr_cnt, cap, ncut_max, ndamp_max, gstride, G,
                                  reinterpret_cast<float *>(smem4));
}

// ------------------------------------------------------------------ networks (FP32)

// One warp per atom: forward pass, atomic energy, and the input gradient
// dE/dG = outw d_L W_L ... d_0 W_0 diag(inpw) (DODZ::grad).
// ------------------------------------------------------------------ FP64 symmetry functions
#define NNP_PI_D 3.141592653589793
//
// NNP::compute_symm (nnp/nnp.cpp:350-392) with every term and sum in FP64,
// for potentials whose input scaling amplifies the FP32 rounding of the
// terms (nnp_set_accumulation(NNP_SYMM_FP64)).  The displacement of each
// neighbour is recovered in FP64 from the wrapped positions: the FP32 record
// d32 = x_i - x_j - R q fixes the integer image q = round(B (x_i - x_j - d32)).
// The basis functions are the FP64 formulas of Cutoff::cutf
// (cutoff.cpp:62-114), BasisR::symmf (basis_radial.cpp:175-257) and
// BasisA::symmf (basis_angular.cpp:212-260), the GAUSS damping width shared
// by a run of equal eta as in BasisA::init (basis_angular.cpp:178-205).
// One warp per atom; the rows are stored as FP32.

__device__ __forceinline__ double cutf64(int name, double r, double rc)
{
    if (!(r < rc)) return 0.0;
    switch (name) {
    case CUT_STEP: return 1.0;
    case CUT_COS: return 0.5 * (cospi(r / rc) + 1.0);
    case CUT_TANH: { const double t = tanh(1.0 - r / rc); return t * t * t; }
    case CUT_POLY3: { const double x = r / rc; return (2.0 * x - 3.0) * x * x + 1.0; }
    default: return 0.0;
    }
}

__device__ __forceinline__ double radial64(int form, double r, double rs, double eta, double fc)
{
    const double x = eta * (r - rs);
    switch (form) {
    case RAD_GAUSSIAN: return exp(-x * x) * fc;
    case RAD_SECH: { const double e = exp(-fabs(x)); return 2.0 * e / (1.0 + e * e) * fc; }
    case RAD_LOGISTIC: { const double e = exp(-fabs(x)), s = 2.0 * e / (1.0 + e * e); return s * s * fc; }
    case RAD_TANH: return 0.5 * (tanh(-x) + 1.0) * fc;
    case RAD_LOGCOSH: {
        const double y = -2.0 * x;
        return 0.5 * ((y > 0.0) ? y + log1p(exp(-y)) : log1p(exp(y))) * fc;
    }
    case RAD_LOGCOSH2: {
        const double k = 2.0 * 1.4142135623730951, a = -x;
        const double f = (fabs(a) < 1e-6) ? 1.0 / k + 0.5 * a + k * a * a / 12.0 : a / (-expm1(-k * a));
        return f * fc;
    }
    default: return 0.0;
    }
}

__device__ __forceinline__ double ipow64(double x, int n)
{
    double r = 1.0;
    while (n) {
        if (n & 1) r *= x;
        x *= x;
        n >>= 1;
    }
    return r;
}

// (lf, zeta, ieta2) of one angular function: value for a pair with cosine cs,
// r_j^2 + r_k^2 = r2s and cutoff product cc
__device__ __forceinline__ double angular64(int form, double cs, double r2s, double cc, double lf, double zeta,
                                            double ieta2)
{
    const double cw = fabs(0.5 + lf * cs);
    const double pz = (zeta == floor(zeta) && zeta >= 0.0 && zeta <= 64.0) ? ipow64(cw, (int)zeta) : pow(cw, zeta);
    double rad;
    switch (form) {
    case ANG_GAUSS: rad = exp(-ieta2 * r2s); break;
    case ANG_GAUSS2: { const double fd = exp(-0.5 * NNP_PI_D * ieta2 * r2s); rad = 2.0 * fd / (1.0 + fd); } break;
    case ANG_SECH: { const double fd = exp(-0.5 * NNP_PI_D * ieta2 * r2s); rad = 2.0 * fd / (1.0 + fd * fd); } break;
    case ANG_STUDENT3: case ANG_STUDENT4: case ANG_STUDENT5:
        rad = ipow64(1.0 / sqrt(1.0 + ieta2 * r2s), 4 + (form - ANG_STUDENT3));
        break;
    default: rad = 0.0;
    }
    return pz * rad * cc;
}

__device__ __forceinline__ double warp_sum64(double v)
{
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
    return v;
}

// shared memory per warp: r, ux, uy, uz and NNP_MAX_CUT cutoff values per
// neighbour slot (doubles), then the neighbour's type (int)
__host__ __device__ inline size_t symm64_floats(int cap) { return (size_t)cap * (2 * (4 + NNP_MAX_CUT) + 1) + 8; }

__global__ void __launch_bounds__(WARPS * 32) k_symm_f64(int64_t N, const DevPot *__restrict__ pot,
                                                          const double2 *__restrict__ rpar64,
                                                          const double4 *__restrict__ apar64,
                                                          const double *__restrict__ cut_rc,
                                                          const int *__restrict__ type, const int *__restrict__ order,
                                                          const float4 *__restrict__ nbr,
                                                          const int *__restrict__ nbr_cnt, int cap,
                                                          const double *__restrict__ xw,
                                                          const int *__restrict__ atom_struct,
                                                          const StructGrid *__restrict__ grid, int gstride,
                                                          float *__restrict__ G)
{
    extern __shared__ double sm64[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double *base = sm64 + (size_t)warp * (symm64_floats(cap) / 2 + 4);
    double *R = base, *UX = R + cap, *UY = UX + cap, *UZ = UY + cap, *FC = UZ + cap;   // FC[c * cap + k]
    int *TY = reinterpret_cast<int *>(FC + NNP_MAX_CUT * cap);
    const DevPot &P = *pot;
    for (int64_t idx = blockIdx.x * (int64_t)WARPS + warp; idx < N; idx += (int64_t)gridDim.x * WARPS) {
        const int64_t i = order[idx];
        const int II = type[i];
        if ((unsigned)II >= (unsigned)P.ntypes) continue;
        const DevType &T = P.t[II];
        const int n = min(nbr_cnt[i], cap);
        const StructGrid &g = grid[atom_struct[i]];
        const double xi0 = xw[3 * i], xi1 = xw[3 * i + 1], xi2 = xw[3 * i + 2];
        for (int k = lane; k < n; k += 32) {
            const float4 rec = nbr[i * cap + k];
            const int jt = __float_as_int(rec.w), j = jt & 0x0fffffff;
            const double sx = xi0 - xw[3 * (int64_t)j], sy = xi1 - xw[3 * (int64_t)j + 1],
                         sz = xi2 - xw[3 * (int64_t)j + 2];
            double dx = sx, dy = sy, dz = sz;
            if (g.pbc) {
                const double ex = sx - rec.x, ey = sy - rec.y, ez = sz - rec.z;     // R q
                double q[3];
                for (int m = 0; m < 3; ++m) q[m] = rint(g.B[3 * m] * ex + g.B[3 * m + 1] * ey + g.B[3 * m + 2] * ez);
                dx -= g.R[0] * q[0] + g.R[3] * q[1] + g.R[6] * q[2];
                dy -= g.R[1] * q[0] + g.R[4] * q[1] + g.R[7] * q[2];
                dz -= g.R[2] * q[0] + g.R[5] * q[1] + g.R[8] * q[2];
            }
            const double r = sqrt(dx * dx + dy * dy + dz * dz);
            R[k] = r;
            UX[k] = dx / r;
            UY[k] = dy / r;
            UZ[k] = dz / r;
            for (int c = 0; c < P.ncut; ++c) FC[c * cap + k] = cutf64(P.cut[c].name, r, cut_rc[c]);
            TY[k] = jt >> 28;
        }
        __syncwarp();
        // neighbours are grouped by type: segment [s0, s1) of type J
        int seg[NNP_MAX_TYPES + 1];
        {
            int c = 0;
            for (int J = 0; J < P.ntypes; ++J) {
                seg[J] = c;
                int cnt = 0;
                for (int k = lane; k < n; k += 32) cnt += (TY[k] == J);
                c += __reduce_add_sync(FULL, cnt);
            }
            seg[P.ntypes] = c;
        }
        float *Gi = G + i * (int64_t)gstride;
        for (int q = lane; q < gstride; q += 32) Gi[q] = 0.f;
        __syncwarp();
        // radial: lane f sums function f over the block's neighbours
        for (int J = 0; J < P.ntypes; ++J) {
            const DevBlockR B = T.br[J];
            if (lane < B.n) {
                const double2 q = rpar64[B.par + lane];
                double acc = 0.0;
                for (int k = seg[J]; k < seg[J + 1]; ++k)
                    acc += radial64(B.form, R[k], q.x, q.y, FC[B.cut * cap + k]);
                Gi[B.off_g + lane] = (float)acc;
            }
        }
        // angular blocks tt = K (K + 1) / 2 + J, J <= K: lanes over the partner b of each first member a
        for (int K = 0, tt = 0; K < P.ntypes; ++K)
            for (int J = 0; J <= K; ++J, ++tt) {
                const DevBlockA B = T.ba[tt];
                if (B.n == 0) continue;
                double acc[NNP_MAX_AFUNC];
                for (int f = 0; f < B.n; ++f) acc[f] = 0.0;
                for (int a = seg[J]; a < seg[J + 1]; ++a) {
                    const int b0 = (J == K) ? a + 1 : seg[K];
                    for (int b = b0 + lane; b < seg[K + 1]; b += 32) {
                        const double cs = UX[a] * UX[b] + UY[a] * UY[b] + UZ[a] * UZ[b];
                        const double r2s = R[a] * R[a] + R[b] * R[b];
                        const double cc = FC[B.cut * cap + a] * FC[B.cut * cap + b];
                        for (int f = 0; f < B.n; ++f) {
                            const double4 q = apar64[B.par + f];
                            acc[f] += angular64(B.form, cs, r2s, cc, q.x, q.y, q.z);
                        }
                    }
                }
                for (int f = 0; f < B.n; ++f) {
                    const double v = warp_sum64(acc[f]);
                    if (lane == 0) Gi[B.off_g + f] = (float)v;
                }
            }
        __syncwarp();
    }
}

__global__ void __launch_bounds__(WARPS * 32) k_nn_fp32(int64_t N, const DevPot *__restrict__ pot,
                                                       const float *__restrict__ wpar, int64_t wfloats,
                                                       const int *__restrict__ type, const float *__restrict__ G,
                                                       int gstride, int maxn, float *__restrict__ e_atom,
                                                       float *__restrict__ dEdG)
{
    extern __shared__ float smem[];
    float *w_s = smem;
    for (int64_t k = threadIdx.x; k < wfloats; k += blockDim.x) w_s[k] = wpar[k];
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float *ws = smem + ((wfloats + 3) & ~3) + (size_t)warp * (NNP_MAX_LAYERS + 2) * maxn;
    float *xa = ws;                      // activations (ping)
    float *xb = ws + maxn;               // activations (pong)
    float *dd = ws + 2 * maxn;           // f'(z) per layer [nlayer][maxn]
    const DevPot &P = *pot;
    for (int64_t i = blockIdx.x * (int64_t)WARPS + warp; i < N; i += (int64_t)gridDim.x * WARPS) {
        const DevType &T = P.t[type[i]];
        const NetView V = net_view(w_s + T.woff, T);
        const int L = T.nlayer, nin = T.nodes[0];
        const float *Gi = G + i * gstride;
        for (int m = lane; m < nin; m += 32) xa[m] = V.inpw[m] * (Gi[m] + V.inpb[m]);
        __syncwarp();
        float *x = xa, *y = xb;
        for (int l = 0; l < L; ++l) {
            const int ni = T.nodes[l], no = T.nodes[l + 1], s = V.ws[l];
            const int neu = (l == L - 1) ? NEU_LINEAR : T.neuron;
            for (int n = lane; n < no; n += 32) {
                float z = V.b[l][n];
                const float *wc = V.wt[l] + n;
                for (int m = 0; m < ni; ++m) z += wc[m * s] * x[m];
                float a, d, d2;
                activation(neu, T.c, z, a, d, d2);
                y[n] = a;
                dd[l * maxn + n] = d;
            }
            __syncwarp();
            float *tmp = x; x = y; y = tmp;
        }
        if (lane == 0) e_atom[i] = V.outb[0] + x[0] * V.outw[0];
        // backward: delta_L = outw * d_L, delta_{l-1} = (W_l^T delta_l) * d_{l-1}
        if (lane == 0) y[0] = V.outw[0] * dd[(L - 1) * maxn];
        __syncwarp();
        float *dl = y, *dn = x;
        for (int l = L - 1; l >= 1; --l) {
            const int ni = T.nodes[l], no = T.nodes[l + 1], s = V.ws[l];
            for (int m = lane; m < ni; m += 32) {
                const float *wr = V.wt[l] + m * s;
                float t = 0.f;
                for (int n = 0; n < no; ++n) t += wr[n] * dl[n];
                dn[m] = t * dd[(l - 1) * maxn + m];
            }
            __syncwarp();
            float *tmp = dl; dl = dn; dn = tmp;
        }
        {
            const int no = T.nodes[1], s = V.ws[0];
            float *out = dEdG + i * gstride;
            for (int m = lane; m < nin; m += 32) {
                const float *wr = V.wt[0] + m * s;
                float t = 0.f;
                for (int n = 0; n < no; ++n) t += wr[n] * dl[n];
                out[m] = t * V.inpw[m];
            }
        }
        __syncwarp();
    }
}

// ------------------------------------------------------------------ forces

__global__ void __launch_bounds__(WARPS * 32, 1) k_force(int64_t N, const DevPot *__restrict__ pot,
                                                        const float2 *__restrict__ rpar, const float4 *__restrict__ apar,
                                                        const int *__restrict__ type, const int *__restrict__ order, const float4 *__restrict__ nbr,
                                                        const int *__restrict__ nbr_cnt, int cap, int ncut_max, int ndamp_max,
                                                        int gstride, const float *__restrict__ dEdG,
                                                        double *__restrict__ F, DevErr *err,
                                                        const int *__restrict__ atom_struct, double *__restrict__ vir)
{
    extern __shared__ float4 smem4[];
    force_body<GenericBlocks>(N, pot, rpar, apar, type, order, nbr, nbr_cnt, cap, ncut_max, ndamp_max, gstride, dEdG, F, err,
                              reinterpret_cast<float *>(smem4), atom_struct, vir);
}

// ------------------------------------------------------------------ energies

__global__ void k_energy(const int64_t *__restrict__ off, int64_t n_centre, const float *__restrict__ e_atom,
                         const int *__restrict__ type, const DevPot *__restrict__ pot, int vacuum,
                         const double *__restrict__ vac, double *__restrict__ e_struct, DevErr *err)
{
    __shared__ double part[256];
    const int s = blockIdx.x;
    double sum = 0.0;
    const int64_t a1 = off[s + 1] < n_centre ? off[s + 1] : n_centre;     // ghosts carry no energy
    for (int64_t a = off[s] + threadIdx.x; a < a1; a += blockDim.x) {
        sum += (double)e_atom[a];
        if (vacuum) {
            const int t = type[a];
            if (t >= 0 && t < pot->ntypes) sum += vac[t];
        }
    }
    part[threadIdx.x] = sum;
    __syncthreads();
    for (int d = blockDim.x / 2; d; d >>= 1) {
        if (threadIdx.x < d) part[threadIdx.x] += part[threadIdx.x + d];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        e_struct[s] = part[0];
        if (!isfinite(part[0])) atomicMax(&err->nonfinite, 1);
    }
}

__global__ void k_nbr_types(int64_t N, const float4 *__restrict__ nbr, const int *__restrict__ nbr_cnt, int cap,
                            int ntypes, int *__restrict__ counts)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= N) return;
    int c[NNP_MAX_TYPES] = {0};
    const int n = nbr_cnt[i];
    for (int k = 0; k < n; ++k) {
        const unsigned t = (unsigned)__float_as_int(nbr[i * cap + k].w) >> 28;
        if (t < NNP_MAX_TYPES) c[t]++;
    }
    for (int t = 0; t < ntypes; ++t) counts[i * ntypes + t] = c[t];
}

std::string run_neighbor_counts(Engine &E, int *d_counts)
{
    if (E.n_atoms == 0) return "";
    k_nbr_types<<<grid_for(E.n_atoms, 256, 1 << 30), 256, 0, E.stream>>>(E.n_atoms, E.nbr.p, E.nbr_cnt.p, E.cap,
                                                                         E.dpot.ntypes, d_counts);
    return cuda_msg("neighbour counts");
}

__global__ void k_f2d(int64_t n, const float *__restrict__ a, double *__restrict__ b)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) b[i] = (double)a[i];
}

__global__ void k_d2f(int64_t n, const double *__restrict__ a, float *__restrict__ b)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) b[i] = (float)a[i];
}

// ------------------------------------------------------------------ host launch sequence

static int num_sms()
{
    static int n = 0;
    if (!n) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (n <= 0) n = 148;
    }
    return n;
}

static int ncut_max(const Engine &E) { return E.dpot.ncut > 0 ? E.dpot.ncut : 1; }

static int ndamp_max(const Engine &E)
{
    int m = 1;
    for (int t = 0; t < E.dpot.ntypes; ++t) m = std::max(m, E.dpot.t[t].ndamp);
    return m;
}

// shared memory of the per-atom kernels; the force view's coefficient arrays
// follow the chunk of the kernel launched (the specialised one's tuned chunk)
static size_t view_bytes(const Engine &E, bool force, bool jit)
{
    const int per = nbr_view_floats(E.cap, ncut_max(E), ndamp_max(E), E.gstride, force,
                                    jit ? E.tune.force_chunk : NNP_PCH);
    return (size_t)WARPS * ((per + 3) & ~3) * sizeof(float);
}

std::string run_prepare(Engine &E, int64_t n_atoms, int n_struct, int pbc)
{
    (void)pbc;
    E.n_atoms = n_atoms;
    E.n_centre = n_atoms - std::min<int64_t>(std::max<int64_t>(E.n_ghost, 0), n_atoms);
    E.n_struct = n_struct;
    const size_t N = (size_t)std::max<int64_t>(n_atoms, 1), S = (size_t)std::max(n_struct, 1);
    const size_t cell_bound = 64 * S + 2 * N + 64;
    cudaError_t e = cudaSuccess;
    auto r = [&](cudaError_t x) { if (x != cudaSuccess && e == cudaSuccess) e = x; };
    r(E.xw.reserve(3 * N));
    r(E.atom_struct.reserve(N));
    r(E.atom_cell.reserve(N));
    r(E.grid.reserve(S));
    r(E.bbox.reserve(6 * S));
    r(E.scan_tmp.reserve(S));
    r(E.cell_cnt.reserve(cell_bound));
    r(E.cell_start.reserve(cell_bound));
    r(E.cell_fill.reserve(cell_bound));
    r(E.cell_tcnt.reserve(cell_bound * (size_t)std::max(E.dpot.ntypes, 1)));
    r(E.cell_atoms.reserve(N));
    r(E.cell_pos.reserve(N));
    r(E.order.reserve(N));
    r(E.type_fill.reserve(NEIGH_ITEM_COUNTER + 1));
    r(E.neigh_items.reserve(N + (N + NEIGH_WARPS - 1) / NEIGH_WARPS + 1));   // parts: at most one per cell and one per warp's atom
    r(E.nbr.reserve(N * (size_t)E.cap));
    r(E.nbr_cnt.reserve(N));
    r(E.G.reserve(N * (size_t)E.gstride));
    r(E.dEdG.reserve(N * (size_t)E.gstride));
    r(E.e_atom.reserve(N));
    r(E.e_struct.reserve(S));
    r(E.force.reserve(3 * N));
    r(E.err.reserve(1));
    if (e != cudaSuccess) return std::string("device allocation failed: ") + cudaGetErrorString(e);
    cudaMemsetAsync(E.err.p, 0, sizeof(DevErr), E.stream);
    return cuda_msg("prepare");
}

std::string run_neighbors(Engine &E, int pbc)
{
    const int64_t N = E.n_atoms;
    const int S = E.n_struct;
    if (N == 0 || S == 0) return "";
    cudaStream_t st = E.stream;
    E.mark(0);
    const size_t cell_bound = 64 * (size_t)S + 2 * (size_t)N + 64;
    // candidate tests per work item: about half a block's share of the
    // search, estimated at 432 tests per atom (27 cells of 16 atoms)
    const int nblocks = num_sms() * NEIGH_BLOCKS;
    const int budget = (int)std::min<int64_t>(1 << 16, std::max<int64_t>(2048, N * 216 / nblocks));
    int *items_n = E.type_fill.p + NEIGH_ITEM_COUNTER;
    const double rc2 = E.dpot.rc_d * E.dpot.rc_d;
    const int nsm = sizeof(NeighShared);
    cudaFuncSetAttribute(k_neigh, cudaFuncAttributeMaxDynamicSharedMemorySize, nsm);
    if (pbc && N <= PRO_MAX_ATOMS && S <= PRO_MAX_STRUCT) {
        // a small periodic batch: the whole prologue in one block
        E.launches += 2;
        k_prologue_small<<<1, PRO_THREADS, 0, st>>>(
            N, E.n_centre, S, (int)cell_bound, E.atom_off.p, E.pos.p, E.cell.p, E.type.p, E.dpot.ntypes,
            E.dpot.rc_d, budget, E.grid.p, E.scan_tmp.p, E.atom_struct.p, E.xw.p, E.atom_cell.p, E.cell_cnt.p,
            E.cell_start.p, E.cell_fill.p, E.cell_atoms.p, E.cell_tcnt.p, E.cell_pos.p, E.type_fill.p, E.order.p,
            E.neigh_items.p, E.err.p);
    } else {
        E.launches += 11;
        cudaMemsetAsync(E.type_fill.p, 0, (NEIGH_ITEM_COUNTER + 1) * sizeof(int), st);
        k_type_count<<<grid_for(N, 256, 1 << 30), 256, 0, st>>>(N, E.n_centre, E.type.p, E.dpot.ntypes, E.type_fill.p);
        k_type_scatter<<<grid_for(N, 256, 1 << 30), 256, 0, st>>>(N, E.n_centre, E.type.p, E.dpot.ntypes, E.type_fill.p,
                                                                   E.type_fill.p + NNP_MAX_TYPES + 1, E.order.p);
        k_atom_struct<<<grid_for(N, 256, 1 << 30), 256, 0, st>>>(E.atom_off.p, S, N, E.atom_struct.p, E.type.p,
                                                                 E.dpot.ntypes, E.err.p);
        if (!pbc) k_struct_bbox<<<S, 256, 0, st>>>(E.pos.p, E.atom_off.p, E.bbox.p);
        k_struct_setup<<<grid_for(S, 128, 1 << 30), 128, 0, st>>>(E.cell.p, E.atom_off.p, S, pbc, E.dpot.rc_d,
                                                                  E.bbox.p, E.grid.p, E.scan_tmp.p, E.err.p);
        E.launches += pbc ? 0 : 1;
        k_cell_base<<<1, 1024, 0, st>>>(E.scan_tmp.p, S, E.grid.p);
        cudaMemsetAsync(E.cell_cnt.p, 0, cell_bound * sizeof(int), st);
        k_bin<<<grid_for(N, 256, 1 << 30), 256, 0, st>>>(N, E.pos.p, E.atom_struct.p, E.grid.p, E.xw.p, E.atom_cell.p,
                                                         E.cell_cnt.p);
        k_cell_start<<<S, 256, 0, st>>>(E.grid.p, E.scan_tmp.p, E.cell_cnt.p, E.cell_start.p, E.cell_fill.p, E.atom_off.p);
        k_fill<<<grid_for(N, 256, 1 << 30), 256, 0, st>>>(N, E.atom_cell.p, E.cell_start.p, E.cell_fill.p, E.cell_atoms.p);
        // (atom_cell, read only by k_fill, holds the keys of the largest cells)
        k_sort_cells<<<num_sms() * 16, SORT_WARPS * 32, 0, st>>>(
            S, E.grid.p, E.scan_tmp.p, E.cell_cnt.p, E.cell_start.p, E.type.p, E.atom_struct.p, E.dpot.ntypes, budget,
            E.cell_atoms.p, E.cell_tcnt.p, reinterpret_cast<unsigned *>(E.atom_cell.p), E.neigh_items.p, items_n);
        k_cell_pos<<<grid_for(N, 256, 1 << 30), 256, 0, st>>>(N, E.cell_atoms.p, E.xw.p, E.type.p, E.dpot.ntypes,
                                                              E.cell_pos.p);
    }
    k_neigh<<<nblocks, NEIGH_THREADS, nsm, st>>>(E.neigh_items.p, items_n, E.grid.p, E.cell_pos.p,
                                                       E.cell_cnt.p, E.cell_start.p, E.cell_tcnt.p, E.cell_atoms.p,
                                                       rc2, E.cap, E.dpot.ntypes, E.nbr.p, E.nbr_cnt.p, E.err.p);
    E.mark(1);
    return cuda_msg("neighbour list");
}

std::string run_symm(Engine &E)
{
    const int64_t N = E.n_centre;      // centres: the first n_centre entries of `order`
    if (N == 0) return "";
    const size_t sm = view_bytes(E, false, false);
    const int grid = grid_for(N, WARPS, num_sms() * 16);
    E.launches += 1;
    if (E.use_jit && E.jit_symm && !E.acc64 && !E.symm64) {
        long long n = N;
        int cap = E.cap, nc = ncut_max(E), nd = ndamp_max(E), gs = E.gstride;
        void *args[] = {&n, &E.d_pot, &E.rpar.p, &E.apar.p, &E.type.p, &E.order.p, &E.nbr.p, &E.nbr_cnt.p,
                        &cap, &nc, &nd, &gs, &E.G.p};
        std::string msg = jit_launch(E.jit_symm, grid, WARPS * 32, sm, E.stream, args);
        E.mark(2);
        return msg;
    }
    if (E.symm64) {
        const size_t sm64 = (size_t)WARPS * (symm64_floats(E.cap) / 2 + 4) * sizeof(double);
        cudaFuncSetAttribute(k_symm_f64, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm64);
        k_symm_f64<<<grid, WARPS * 32, sm64, E.stream>>>(N, E.d_pot, E.rpar64.p, E.apar64.p, E.cut64.p, E.type.p,
                                                         E.order.p, E.nbr.p, E.nbr_cnt.p, E.cap, E.xw.p,
                                                         E.atom_struct.p, E.grid.p, E.gstride, E.G.p);
        E.mark(2);
        return cuda_msg("symmetry functions (FP64)");
    }
    auto kern = E.acc64 ? k_symm<double> : k_symm<float>;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    kern<<<grid, WARPS * 32, sm, E.stream>>>(N, E.d_pot, E.rpar.p, E.apar.p, E.type.p, E.order.p, E.nbr.p, E.nbr_cnt.p, E.cap,
                                             ncut_max(E), ndamp_max(E), E.gstride, E.G.p);
    E.mark(2);
    return cuda_msg("symmetry functions");
}

static int max_nodes(const Engine &E)
{
    int m = 1;
    for (int t = 0; t < E.dpot.ntypes; ++t)
        for (int l = 0; l <= E.dpot.t[t].nlayer; ++l) m = std::max(m, E.dpot.t[t].nodes[l]);
    return (m + 3) & ~3;
}

std::string run_nn(Engine &E)
{
    const int64_t N = E.n_atoms;
    if (N == 0) return "";
    // BF16 / split-BF16 tensor-core layers when every network fits them
    if (E.precision != NNP_PREC_FP32 && tc_smem_bytes(E, E.precision == NNP_PREC_BF16X3) > 0)
        return run_nn_tc(E, E.precision == NNP_PREC_BF16X3);
    const int maxn = max_nodes(E);
    const size_t sm = (size_t)(((E.wfloats + 3) & ~3) + WARPS * (NNP_MAX_LAYERS + 2) * maxn) * sizeof(float);
    if (sm > 220 * 1024) return "networks too large for the shared-memory FP32 path";
    cudaFuncSetAttribute(k_nn_fp32, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k_nn_fp32<<<grid_for(N, WARPS * 8, num_sms() * 2), WARPS * 32, sm, E.stream>>>(
        E.n_centre, E.d_pot, E.wpar.p, E.wfloats, E.type.p, E.G.p, E.gstride, maxn, E.e_atom.p, E.dEdG.p);
    E.launches += 1;
    E.mark(3);
    return cuda_msg("networks");
}

std::string run_force(Engine &E)
{
    const int64_t N = E.n_centre;      // centres; forces are scattered onto every atom, ghosts included
    if (E.n_atoms == 0) return "";
    cudaMemsetAsync(E.force.p, 0, 3 * (size_t)E.n_atoms * sizeof(double), E.stream);
    double *vir = E.want_virial ? E.vir.p : nullptr;
    if (vir) cudaMemsetAsync(vir, 0, 9 * (size_t)E.n_struct * sizeof(double), E.stream);
    const size_t sm = view_bytes(E, true, E.use_jit && E.jit_force);
    const int grid = grid_for(N, WARPS, num_sms() * 16);
    E.launches += 1;
    if (E.use_jit && E.jit_force) {
        long long n = N;
        int cap = E.cap, nc = ncut_max(E), nd = ndamp_max(E), gs = E.gstride;
        void *args[] = {&n, &E.d_pot, &E.rpar.p, &E.apar.p, &E.type.p, &E.order.p, &E.nbr.p, &E.nbr_cnt.p,
                        &cap, &nc, &nd, &gs, &E.dEdG.p, &E.force.p, &E.err.p, &E.atom_struct.p, &vir};
        std::string msg = jit_launch(E.jit_force, grid, WARPS * 32, sm, E.stream, args);
        E.mark(4);
        return msg;
    }
    cudaFuncSetAttribute(k_force, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k_force<<<grid, WARPS * 32, sm, E.stream>>>(N, E.d_pot, E.rpar.p, E.apar.p, E.type.p, E.order.p, E.nbr.p, E.nbr_cnt.p, E.cap,
                                                ncut_max(E), ndamp_max(E), E.gstride, E.dEdG.p, E.force.p, E.err.p,
                                                E.atom_struct.p, vir);
    E.mark(4);
    return cuda_msg("forces");
}

std::string run_energy(Engine &E, bool vacuum)
{
    if (E.n_struct == 0) return "";
    k_energy<<<E.n_struct, 256, 0, E.stream>>>(E.atom_off.p, E.n_centre, E.e_atom.p, E.type.p, E.d_pot, vacuum ? 1 : 0,
                                               E.vac.p, E.e_struct.p, E.err.p);
    E.launches += 1;
    E.mark(5);
    return cuda_msg("energies");
}

// per-atom energies in FP64: the network energy of each atom, plus its
// element's vacuum energy when requested (NNH::energy, nnh.cpp:207-210)
__global__ void k_atom_energy(int64_t N, const float *__restrict__ e_atom, const int *__restrict__ type, int ntypes,
                              int vacuum, const double *__restrict__ vac, double *__restrict__ out)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= N) return;
    const int t = type[i];
    out[i] = (double)e_atom[i] + ((vacuum && t >= 0 && t < ntypes) ? vac[t] : 0.0);
}

std::string run_atom_energy(Engine &E, bool vacuum, double *out)
{
    const int64_t N = E.n_centre;
    if (N == 0) return "";
    k_atom_energy<<<grid_for(N, 256, 1 << 30), 256, 0, E.stream>>>(N, E.e_atom.p, E.type.p, E.dpot.ntypes,
                                                                   vacuum ? 1 : 0, E.vac.p, out);
    E.launches += 1;
    return cuda_msg("per-atom energies");
}

std::string run_symm_to_double(Engine &E, double *out)
{
    const int64_t n = E.n_atoms * E.gstride;
    if (n == 0) return "";
    k_f2d<<<grid_for(n, 256, 1 << 30), 256, 0, E.stream>>>(n, E.G.p, out);
    return cuda_msg("symm copy");
}

std::string run_nn_from_symm(Engine &E, const double *symm_d, int gstride_in)
{
    (void)gstride_in;
    const int64_t n = E.n_atoms * E.gstride;
    if (n == 0) return "";
    k_d2f<<<grid_for(n, 256, 1 << 30), 256, 0, E.stream>>>(n, symm_d, E.G.p);
    return run_nn(E);
}

// ------------------------------------------------------------------ allocation-free energies
//
// Energies of a batch from device-resident symmetry functions for callers
// that must not allocate device memory during the call (a serving loop that
// has reserved all of its memory up front, or one running under an external
// allocator): cudaMalloc/cudaFree synchronise the whole device and can fail
// under memory pressure.  The only scratch, one FP32 energy per atom, lives
// in this file-scope array, so the call's size limit is NNP_NOALLOC_MAX_ATOMS
// atoms.  Every call writes entries [0, N) before it reads them (same
// stream, kernel order), so the array needs no initial contents.  It is one
// array per device, shared by every handle on that device: calls that may
// overlap in time (different streams or host threads) race on it and must be
// ordered by the caller.

static __device__ __align__(256) float g_noalloc_e_atom[NNP_NOALLOC_MAX_ATOMS];

// Forward pass only (the energy half of k_nn_fp32, same arithmetic order);
// an atom whose type is outside [0, ntypes) gets a NaN energy.
__global__ void __launch_bounds__(WARPS * 32) k_nn_energy_fp32(int64_t N, const DevPot *__restrict__ pot,
                                                              const float *__restrict__ wpar, int64_t wfloats,
                                                              const int *__restrict__ type,
                                                              const float *__restrict__ G, int gstride, int maxn,
                                                              float *__restrict__ e_atom)
{
    extern __shared__ float smem[];
    float *w_s = smem;
    for (int64_t k = threadIdx.x; k < wfloats; k += blockDim.x) w_s[k] = wpar[k];
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float *xa = smem + ((wfloats + 3) & ~3) + (size_t)warp * 2 * maxn;
    float *xb = xa + maxn;
    const DevPot &P = *pot;
    for (int64_t i = blockIdx.x * (int64_t)WARPS + warp; i < N; i += (int64_t)gridDim.x * WARPS) {
        const int ti = type[i];
        if (ti < 0 || ti >= P.ntypes) {
            if (lane == 0) e_atom[i] = __int_as_float(0x7fffffff);
            continue;
        }
        const DevType &T = P.t[ti];
        const NetView V = net_view(w_s + T.woff, T);
        const int L = T.nlayer, nin = T.nodes[0];
        const float *Gi = G + i * gstride;
        for (int m = lane; m < nin; m += 32) xa[m] = V.inpw[m] * (Gi[m] + V.inpb[m]);
        __syncwarp();
        float *x = xa, *y = xb;
        for (int l = 0; l < L; ++l) {
            const int ni = T.nodes[l], no = T.nodes[l + 1], s = V.ws[l];
            const int neu = (l == L - 1) ? NEU_LINEAR : T.neuron;
            for (int n = lane; n < no; n += 32) {
                float z = V.b[l][n];
                const float *wc = V.wt[l] + n;
                for (int m = 0; m < ni; ++m) z += wc[m * s] * x[m];
                float a, d, d2;
                activation(neu, T.c, z, a, d, d2);
                y[n] = a;
            }
            __syncwarp();
            float *tmp = x; x = y; y = tmp;
        }
        if (lane == 0) e_atom[i] = V.outb[0] + x[0] * V.outw[0];
        __syncwarp();
    }
}

// One block per structure, FP64 sum (as k_energy); an out-of-range type
// with vacuum energies requested gives NaN, and so does a structure whose
// offsets fall outside [0, N] (nothing outside the N scratch entries is read).
__global__ void k_energy_noalloc(const int64_t *__restrict__ off, int64_t N, const float *__restrict__ e_atom,
                                 const int *__restrict__ type, int ntypes, int vacuum,
                                 const double *__restrict__ vac, double *__restrict__ e_struct)
{
    __shared__ double part[256];
    const int s = blockIdx.x;
    const int64_t a0 = off[s], a1 = off[s + 1];
    if (a0 < 0 || a1 < a0 || a1 > N) {
        if (threadIdx.x == 0) e_struct[s] = __longlong_as_double(0x7ff8000000000000ll);
        return;
    }
    double sum = 0.0;
    for (int64_t a = a0 + threadIdx.x; a < a1; a += blockDim.x) {
        sum += (double)e_atom[a];
        if (vacuum) {
            const int t = type[a];
            sum += (t >= 0 && t < ntypes) ? vac[t] : __longlong_as_double(0x7ff8000000000000ll);
        }
    }
    part[threadIdx.x] = sum;
    __syncthreads();
    for (int d = blockDim.x / 2; d; d >>= 1) {
        if (threadIdx.x < d) part[threadIdx.x] += part[threadIdx.x + d];
        __syncthreads();
    }
    if (threadIdx.x == 0) e_struct[s] = part[0];
}

// Device address of the scratch array on the handle's device, looked up on
// the handle's first allocation-free call (cudaGetSymbolAddress may load the
// module; it allocates nothing the caller owns) and kept with the handle: a
// handle lives in one CUDA context, so the address cannot go stale under it
// (a handle made after a device reset looks it up again).
std::string noalloc_scratch(Engine &E, float **out)
{
    if (!E.noalloc_e_atom) {
        float *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress((void **)&p, g_noalloc_e_atom);
        if (e != cudaSuccess) return std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e);
        E.noalloc_e_atom = p;
    }
    *out = E.noalloc_e_atom;
    return "";
}

std::string run_energy_symm_noalloc(Engine &E, int S, int64_t N, const int64_t *off, const int *type,
                                    const float *G, int gstride, bool vacuum, double *energy)
{
    float *e_atom = nullptr;
    std::string msg = noalloc_scratch(E, &e_atom);
    if (!msg.empty()) return msg;
    if (S == 0) return "";
    const int maxn = max_nodes(E);
    const size_t sm = (size_t)(((E.wfloats + 3) & ~3) + WARPS * 2 * maxn) * sizeof(float);
    if (sm > 220 * 1024) return "networks too large for the shared-memory FP32 path";
    if (N > 0) {
        cudaError_t e = cudaFuncSetAttribute(k_nn_energy_fp32, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e != cudaSuccess) return std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e);
        k_nn_energy_fp32<<<grid_for(N, WARPS * 8, num_sms() * 2), WARPS * 32, sm, E.stream>>>(
            N, E.d_pot, E.wpar.p, E.wfloats, type, G, gstride, maxn, e_atom);
        E.launches += 1;
    }
    k_energy_noalloc<<<S, 256, 0, E.stream>>>(off, N, e_atom, type, E.dpot.ntypes, vacuum ? 1 : 0, E.vac.p, energy);
    E.launches += 1;
    return cuda_msg("allocation-free energies");
}

}  // namespace nnp
