// pq_laplace_bc.cu -- the Dirichlet boundary routines of qg_laplace_bc
// (qg3p_laplace_bc.F90:14-374) as device kernels behind the C ABI:
// add_laplace_bc_rhs (the right-hand-side lifting of a boundary value into
// the rows and columns next to the boundary), laplace_bc_rhs (the same on a
// zero field) and apply_dirichlet_bc (the boundary values themselves), for
// the closed basin and the channel, one layer or several with one value or
// one per layer.
//
// Both kernels touch O(perimeter) nodes.  One thread owns one node and
// applies, in the reference's order, every subtraction the reference's
// loops make there (a corner of the lifting ring is lowered twice, as the
// reference does), so the results match the reference bit for bit.
#include <cuda_runtime.h>

#include <cstring>

#include "pq_ctx.h"

namespace {

struct BcValues {
    double b[PQ_MAX_LAYERS];  // closed basin: every wall; channel: wall i = 1
    double d[PQ_MAX_LAYERS];  // channel: wall i = ii
};

// Lifting ring of one layer (0-based node indices).  Closed basin
// (qg3p_laplace_bc.F90:55-86): rows j = 1 and j = jj-2 over i = 1..ii-2 and
// columns i = 1 and i = ii-2 over the rows between; each node subtracts bc
// once per ring side it lies on, in the order j = l_j_max, j = l_j_min,
// i = l_i_min, i = l_i_max.  Channel (:128-150): columns i = 1 (bc_b) and
// i = ii-2 (bc_d) over every row.
__global__ void k_add_laplace_bc_rhs(double* f, int ii, int jj, int pitch, size_t plane, int periodic,
                                     BcValues v) {
    const int l = blockIdx.y;
    const double bb = v.b[l], bd = v.d[l];
    double* p = f + plane * l;
    const int imin = 1, imax = ii - 2;
    const int nrow_i = imax - imin + 1;
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (!periodic) {
        const int jmin = 1, jmax = jj - 2;
        const int nrows = jmax > jmin ? 2 : 1;
        const long n_rows = (long)nrows * nrow_i;
        const int ncol = imax > imin ? 2 : 1;
        const long n_cols = (long)ncol * (jmax - jmin - 1 > 0 ? jmax - jmin - 1 : 0);
        int i, j;
        if (t < n_rows) {
            j = (t / nrow_i) == 0 ? jmin : jmax;
            i = imin + (int)(t % nrow_i);
        } else if (t < n_rows + n_cols) {
            const long u = t - n_rows;
            const int span = jmax - jmin - 1;
            i = (u / span) == 0 ? imin : imax;
            j = jmin + 1 + (int)(u % span);
        } else {
            return;
        }
        double x = p[(size_t)j * pitch + i];
        if (j == jmax) x -= bb;
        if (j == jmin) x -= bb;
        if (i == imin) x -= bb;
        if (i == imax) x -= bb;
        p[(size_t)j * pitch + i] = x;
    } else {
        const int ncol = imax > imin ? 2 : 1;
        if (t >= (long)ncol * jj) return;
        const int i = (t / jj) == 0 ? imin : imax;
        const int j = (int)(t % jj);
        double x = p[(size_t)j * pitch + i];
        if (i == imin) x -= bb;
        if (i == imax) x -= bd;
        p[(size_t)j * pitch + i] = x;
    }
}

// Boundary nodes of one layer (qg3p_laplace_bc.F90:193-224 closed basin:
// every node of rows j = 0, jj-1 and columns i = 0, ii-1 takes bc;
// :227-251 channel: column i = 0 takes bc_b, column i = ii-1 bc_d).  Each
// node is written once.
__global__ void k_apply_dirichlet_bc(double* f, int ii, int jj, int pitch, size_t plane, int periodic, BcValues v) {
    const int l = blockIdx.y;
    const double bb = v.b[l], bd = v.d[l];
    double* p = f + plane * l;
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (!periodic) {
        const long n_rows = 2L * ii;
        const long n_cols = 2L * (jj - 2);
        if (t < n_rows) {
            const int j = (t / ii) == 0 ? 0 : jj - 1;
            p[(size_t)j * pitch + (t % ii)] = bb;
        } else if (t < n_rows + n_cols) {
            const long u = t - n_rows;
            const int i = (u / (jj - 2)) == 0 ? 0 : ii - 1;
            const int j = 1 + (int)(u % (jj - 2));
            p[(size_t)j * pitch + i] = bb;
        }
    } else {
        if (t >= 2L * jj) return;
        const int j = (int)(t % jj);
        if (t / jj == 0)
            p[(size_t)j * pitch] = bb;
        else
            p[(size_t)j * pitch + ii - 1] = bd;
    }
}

enum BcOp { OP_ADD_RHS = 0, OP_APPLY = 1 };

int boundary_op(pq_ctx* c, double* field, int layers, const double* bc, const double* bc_d, int nbc, int kind,
                BcOp op) {
    using pq::fail;
    if (!c || !field || !bc) return PQ_ERR_ARG;
    if (layers < 1 || layers > c->L)
        return fail(c, PQ_ERR_ARG, "layers must be 1..the context's layer count");
    if (nbc != 1 && nbc != layers) return fail(c, PQ_ERR_ARG, "nbc must be 1 or layers");
    if (bc_d && !c->periodic) return fail(c, PQ_ERR_ARG, "bc_d (a second wall value) applies to a channel only");
    if (kind != PQ_PTR_HOST && kind != PQ_PTR_DEVICE) return fail(c, PQ_ERR_ARG, "bad ptr_kind");
    BcValues v;
    std::memset(&v, 0, sizeof(v));
    for (int l = 0; l < layers; ++l) {
        v.b[l] = bc[nbc == 1 ? 0 : l];
        v.d[l] = bc_d ? bc_d[nbc == 1 ? 0 : l] : v.b[l];
    }
    const int ii = c->ii, jj = c->jj;
    CK(cudaSetDevice(c->device));
    // Host arrays go through the context's helm_io field (pitched); device
    // arrays are worked on in place (dense, pitch ii).
    double* dev = field;
    int pitch = ii;
    if (kind == PQ_PTR_HOST) {
        dev = static_cast<double*>(c->hm[0].helm_io);
        pitch = c->pitch;
        const size_t w = (size_t)ii * sizeof(double);
        CK(cudaMemcpy2DAsync(dev, (size_t)pitch * sizeof(double), field, w, w, (size_t)jj * layers,
                             cudaMemcpyHostToDevice, c->stream));
    }
    const size_t plane = (size_t)pitch * jj;
    const long nodes = 2L * ii + 2L * jj;  // covers both kernels' node lists
    const dim3 grid((unsigned)((nodes + 127) / 128), (unsigned)layers);
    if (op == OP_ADD_RHS)
        k_add_laplace_bc_rhs<<<grid, 128, 0, c->stream>>>(dev, ii, jj, pitch, plane, c->periodic ? 1 : 0, v);
    else
        k_apply_dirichlet_bc<<<grid, 128, 0, c->stream>>>(dev, ii, jj, pitch, plane, c->periodic ? 1 : 0, v);
    CK(cudaGetLastError());
    c->last_launches = 1;
    if (kind == PQ_PTR_HOST) {
        const size_t w = (size_t)ii * sizeof(double);
        CK(cudaMemcpy2DAsync(field, w, dev, (size_t)pitch * sizeof(double), w, (size_t)jj * layers,
                             cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
    }
    return PQ_OK;
}

}  // namespace

extern "C" {

int pq_add_laplace_bc_rhs(pq_ctx* c, double* rhs, int layers, const double* bc, const double* bc_d, int nbc,
                          int ptr_kind) {
    return boundary_op(c, rhs, layers, bc, bc_d, nbc, ptr_kind, OP_ADD_RHS);
}

int pq_apply_dirichlet_bc(pq_ctx* c, double* field, int layers, const double* bc, const double* bc_d, int nbc,
                          int ptr_kind) {
    return boundary_op(c, field, layers, bc, bc_d, nbc, ptr_kind, OP_APPLY);
}

int pq_laplace_bc_rhs(pq_ctx* c, double bc, double* rhs, int ptr_kind) {
    if (!c || !rhs) return PQ_ERR_ARG;
    CK(cudaSetDevice(c->device));
    const size_t bytes = (size_t)c->ii * c->jj * sizeof(double);
    if (ptr_kind == PQ_PTR_DEVICE)
        CK(cudaMemsetAsync(rhs, 0, bytes, c->stream));
    else if (ptr_kind == PQ_PTR_HOST)
        std::memset(rhs, 0, bytes);
    else
        return pq::fail(c, PQ_ERR_ARG, "bad ptr_kind");
    return boundary_op(c, rhs, 1, &bc, nullptr, 1, ptr_kind, OP_ADD_RHS);
}

}  // extern "C"
