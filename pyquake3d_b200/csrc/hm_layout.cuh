// Packed H-matrix layout shared by assembly, ACA packing and the matvec.
//
// All row/column indices are positions in cluster-tree order (a depth-first,
// left-first walk of the cluster tree), so every block covers contiguous
// ranges [r0, r0+m) x [c0, c0+n) and the operator needs no gather/scatter.
//
// Column alignment: a block's stored columns start at the CW-aligned column
// c0a = c0 - lead (lead = c0 % CW, zero-filled), so the x slice of a column group
// is one aligned vector load.
//
// Dense block (m x n, six operators): element (row i, col j, comp c, slip s)
//   at  (((jj / CW) * 6 + 2*c + s) * m + i) * CW + (jj % CW),  jj = j + lead
// with comp c in {tau1, tau2, sigma_n} and slip s in {strike, dip}; CW is 4
// for FP32 and 2 for FP64.  For one column group and one operator the rows are
// consecutive 16-byte pieces, so a warp (lanes over rows) loads 512 contiguous
// bytes per instruction.
//
// Low-rank block (ACA): for comp c the block is U_c T_c with
//   U_c = [U_cs | U_cd]  (m x K, K = kS + kD, padded to a multiple of CWU)
//   t_c = [V_cs x_strike ; V_cd x_dip]
// U element (row i, comp c, q) at (((q / CWU) * 3 + c) * m + i) * CWU + q % CWU.
// V rows: Q = 3*kS + 3*kD rows (A1s, A2s, Bs rows first, then A1d, A2d, Bd),
// column-group major: element (q, j) at ((jj / CWV) * Q + q) * CWV + jj % CWV
// with jj = lead + j, so 8 consecutive rows of one column group are 128
// contiguous bytes.
//
// The deficit vector x (accumulation type) holds, with P = x_stride(n):
//   x[0 .. 2P)    interleaved (strike, dip) per element  -- dense blocks
//   x[2P .. 3P)   strike plane, x[3P .. 4P) dip plane     -- V rows
// all zero beyond n.
#pragma once
#include <stdint.h>

namespace pq3d {

constexpr int kCW32 = 4;   // dense FP32 column group
constexpr int kCW64 = 2;   // dense FP64 column group

struct DenseBlock {
    int64_t off64, off32;  // element offsets of the block in the FP64 / FP32 dense arrays
    int32_t m, n, r0, c0;
};

__host__ __device__ inline int64_t dense_index(int m, int i, int j, int comp, int slip, int cw)
{
    return (((int64_t)(j / cw) * 6 + 2 * comp + slip) * m + i) * cw + (j % cw);
}

__host__ __device__ inline int64_t u_index(int m, int i, int comp, int q, int cwu)
{
    return (((int64_t)(q / cwu) * 3 + comp) * m + i) * cwu + (q % cwu);
}

__host__ __device__ inline int64_t v_index(int Q, int q, int jj, int cwv)
{
    return ((int64_t)(jj / cwv) * Q + q) * cwv + (jj % cwv);
}

__host__ __device__ inline int x_stride(int n) { return ((n + 16 + 7) / 8) * 8; }

// Matvec work items (one warp each).
struct DenseItem {          // rows [r, r+32) of a dense block, column groups [g0, g1)
    int64_t off;            // block offset in the dense array
    int32_t m, r, g0, g1, c0, slot;  // slot: slot index of block row 0 for this column chunk
};
struct VItem {              // V rows [q, q+nr) (nr <= 32, one slip) of a block, column groups [g0, g1)
    int64_t off;            // block offset in the V array
    int32_t Q, q, nr, g0, g1, c0, s, tp;  // s: slip of these rows; tp: this chunk's partial t (Q values)
};
struct VItemM {             // mixed storage: rows [rows, rows + nr) (nr <= 32) of the VRowRec list,
    int64_t rows;           // one class and one slip, from the low-rank blocks that share one
    int32_t nr, g0, g1, c0, s, pad;  // column cluster; column groups [g0, g1); s: slip | class << 8
};
struct VRowRec {            // one V row of a VItemM
    int64_t base;           // element offset of (column group 0, this row) in its class array
    int32_t stride;         // elements per column group of its block (Q * CW)
    int32_t out;            // index of this row's chunk partial in t
};
struct UTask {              // one CTA: rows [r0, r1) of a low-rank block
    int64_t off;            // block offset in the U array
    int32_t m, r0, r1, K, kS, kD, Q, tp, nch, slot;  // tp/nch: the block's chunk partials of t (stride Q)
};

}  // namespace pq3d
