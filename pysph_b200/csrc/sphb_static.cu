// sphb_static.cu -- neighbour counting whose scratch lives in the library.
//
// sphb_neighbor_counts_static counts, for every particle of one particle set,
// the particles j with |x_i - x_j|^2 < (radius_scale * h_i)^2 (self included),
// the same FP64 predicate as sphb_neighbors.  It takes only the caller's
// input and output arrays: its cell tables, keys and permutation live in one
// file-scope __device__ array (sphb_static_scratch, SPHB_STATIC_SCRATCH_BYTES,
// held by every GPU that loads this library until the process exits).
//
// Who needs it: callers that cannot call cudaMalloc -- for example a host
// application whose own memory manager owns all device memory and hands this
// library nothing but the particle arrays, or code on a latency-critical path
// where cudaMalloc's implicit device-wide synchronisation is not acceptable.
//
// Set-up: the first call on a device looks up the array's device address
// (cudaGetSymbolAddress, with that device current) and caches it; make that
// first call on each device before any stream capture.  cudaDeviceReset
// unloads the library's device code, so the cached address of that device
// is then stale: the entry point must not be called on a device after it
// was reset.  Every call shares the
// one array and it keeps the last call's contents, so calls that overlap on
// the GPU (different streams, or different host threads, same device) race:
// serialise them.  The call allocates nothing.

#include <mutex>

#include "sphb_common.cuh"
#include "sphb_pairs.cuh"

#define SPHB_STATIC_MAX_CELLS (1 << 19)
#define SPHB_STATIC_HEADER 256
#define SPHB_STATIC_REGION(n) ((((size_t)(n) * 4) + 255) & ~(size_t)255)
#define SPHB_STATIC_SCRATCH_BYTES                                            \
    (SPHB_STATIC_HEADER + SPHB_STATIC_REGION(SPHB_STATIC_MAX_CELLS) +        \
     SPHB_STATIC_REGION(SPHB_STATIC_MAX_CELLS + 1) +                         \
     3 * SPHB_STATIC_REGION(SPHB_STATIC_MAX_PARTICLES))

static __device__ __align__(256) unsigned char sphb_static_scratch[SPHB_STATIC_SCRATCH_BYTES];

namespace sphb {
namespace nalloc {

// Header at the start of the scratch array.
struct Header {
    unsigned long long box[6];   // order-encoded min xyz, max xyz
    unsigned long long hmax;     // bits of max h (>= 0)
    double cs;                   // cell size used
    int lo[3];                   // global cell of local cell (0,0,0)
    int n[3];                    // grid dims
    int ncells;
};

struct View {
    Header *hdr;
    int *count, *start, *key, *slot, *perm;
};

__host__ __device__ inline View carve(unsigned char *base)
{
    View v;
    size_t off = 0;
    v.hdr = (Header *)(base + off);
    off += SPHB_STATIC_HEADER;
    v.count = (int *)(base + off);
    off += SPHB_STATIC_REGION(SPHB_STATIC_MAX_CELLS);
    v.start = (int *)(base + off);
    off += SPHB_STATIC_REGION(SPHB_STATIC_MAX_CELLS + 1);
    v.key = (int *)(base + off);
    off += SPHB_STATIC_REGION(SPHB_STATIC_MAX_PARTICLES);
    v.slot = (int *)(base + off);
    off += SPHB_STATIC_REGION(SPHB_STATIC_MAX_PARTICLES);
    v.perm = (int *)(base + off);
    return v;
}

struct Input {
    int n, dim;
    const double *x, *y, *z, *h;
    double radius_scale;
};

__global__ void k_reset(unsigned char *base)
{
    View v = carve(base);
    if (threadIdx.x < 3) {
        v.hdr->box[threadIdx.x] = enc_double(INFINITY);
        v.hdr->box[3 + threadIdx.x] = enc_double(-INFINITY);
    }
    if (threadIdx.x == 0) v.hdr->hmax = 0ull;
}

__global__ void __launch_bounds__(256) k_bounds(unsigned char *base, Input in)
{
    View v = carve(base);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double p[3] = {0.0, 0.0, 0.0};
    double h = 0.0;
    bool ok = false;
    if (i < in.n) {
        p[0] = in.x[i];
        p[1] = in.y[i];
        if (in.dim == 3) p[2] = in.z[i];
        h = in.h[i];
        ok = isfinite(p[0]) && isfinite(p[1]) && isfinite(p[2]);
    }
    for (int d = 0; d < in.dim; ++d) {
        const double lo = block_reduce(ok ? p[d] : INFINITY, OpMin(), (double)INFINITY);
        if (threadIdx.x == 0 && lo < INFINITY) atomicMin(&v.hdr->box[d], enc_double(lo));
        const double hi = block_reduce(ok ? p[d] : -INFINITY, OpMax(), (double)-INFINITY);
        if (threadIdx.x == 0 && hi > -INFINITY) atomicMax(&v.hdr->box[3 + d], enc_double(hi));
    }
    const double hm = block_reduce(isfinite(h) ? h : 0.0, OpMax(), 0.0);
    if (threadIdx.x == 0) atomic_max_nonneg(&v.hdr->hmax, hm);
}

// Cell size >= radius_scale * max h, doubled until the padded grid fits.
__global__ void k_grid(unsigned char *base, Input in)
{
    View v = carve(base);
    Header &H = *v.hdr;
    double cs = in.radius_scale * __longlong_as_double((long long)H.hmax);
    if (!(cs > 0.0) || !isfinite(cs)) cs = 1.0;
    double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    for (int d = 0; d < in.dim; ++d) {
        lo[d] = dec_double(H.box[d]);
        hi[d] = dec_double(H.box[3 + d]);
        if (!(lo[d] <= hi[d])) lo[d] = hi[d] = 0.0;
    }
    for (int it = 0; it < 200; ++it) {
        long long cells = 1;
        bool fits = true;
        for (int d = 0; d < 3; ++d) {
            if (d < in.dim) {
                const double flo = floor(lo[d] / cs), fhi = floor(hi[d] / cs);
                const double span = fhi - flo + 3.0;
                if (!(span < (double)SPHB_STATIC_MAX_CELLS)) { fits = false; break; }
                // global cell coordinates must fit an int: particles far
                // from the origin against the cell size widen the cells
                if (!(fabs(flo) < 1073741824.0 && fabs(fhi) < 1073741824.0)) {
                    fits = false;
                    break;
                }
                H.lo[d] = (int)flo - 1;
                H.n[d] = (int)span;
            } else {
                H.lo[d] = 0;
                H.n[d] = 1;
            }
            cells *= H.n[d];
            if (cells > SPHB_STATIC_MAX_CELLS) { fits = false; break; }
        }
        if (fits) {
            H.cs = cs;
            H.ncells = (int)cells;
            return;
        }
        cs *= 2.0;
    }
    H.cs = cs;
    H.ncells = 0;  // unreachable for finite boxes; counts become -1
}

// Clears count[0 .. ncells) of the grid k_grid chose (grid-stride: the
// launch does not know ncells).
__global__ void __launch_bounds__(256) k_zero(unsigned char *base)
{
    View v = carve(base);
    const int nc = v.hdr->ncells;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x)
        v.count[c] = 0;
}

__device__ inline int cell_key(const Header &H, double x, double y, double z, int dim)
{
    const double p[3] = {x, y, z};
    int c[3] = {0, 0, 0};
    for (int d = 0; d < dim; ++d) {
        if (!isfinite(p[d])) return -1;
        const double f = floor(p[d] / H.cs) - (double)H.lo[d];
        if (!(f >= 0.0) || !(f < (double)H.n[d])) return -1;
        c[d] = (int)f;
    }
    return (c[2] * H.n[1] + c[1]) * H.n[0] + c[0];
}

__global__ void __launch_bounds__(256) k_hash(unsigned char *base, Input in)
{
    View v = carve(base);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= in.n) return;
    const int key = cell_key(*v.hdr, in.x[i], in.y[i], in.dim == 3 ? in.z[i] : 0.0, in.dim);
    v.key[i] = key;
    if (key >= 0 && key < v.hdr->ncells) v.slot[i] = atomicAdd(&v.count[key], 1);
    else v.key[i] = -1;
}

// One block: exclusive scan of count[0..ncells) into start[0..ncells].
__global__ void __launch_bounds__(1024) k_scan(unsigned char *base)
{
    __shared__ int part[1024];
    View v = carve(base);
    const int T = v.hdr->ncells;
    const int per = (T + blockDim.x - 1) / blockDim.x;
    const int b = threadIdx.x * per;
    const int e = min(T, b + per);
    int s = 0;
    for (int c = b; c < e; ++c) s += v.count[c];
    part[threadIdx.x] = s;
    __syncthreads();
    for (int off = 1; off < (int)blockDim.x; off <<= 1) {
        const int add = (int)threadIdx.x >= off ? part[threadIdx.x - off] : 0;
        __syncthreads();
        part[threadIdx.x] += add;
        __syncthreads();
    }
    int run = part[threadIdx.x] - s;
    for (int c = b; c < e; ++c) {
        v.start[c] = run;
        run += v.count[c];
    }
    if (threadIdx.x == blockDim.x - 1) v.start[T] = part[threadIdx.x];
}

__global__ void __launch_bounds__(256) k_scatter(unsigned char *base, int n)
{
    View v = carve(base);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int key = v.key[i];
    if (key < 0) return;
    const int pos = v.start[key] + v.slot[i];
    if (pos >= 0 && pos < n) v.perm[pos] = i;
}

template <int DIM>
__global__ void __launch_bounds__(256) k_count(unsigned char *base, Input in, int *counts)
{
    View v = carve(base);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= in.n) return;
    const int key = v.key[i];
    // a non-finite position has no cell; a non-finite h no support radius
    if (key < 0 || !isfinite(in.h[i])) {
        counts[i] = -1;
        return;
    }
    const Header &H = *v.hdr;
    int cx, cy, cz;
    cell_coords(key, H.n, cx, cy, cz);
    const double xi = in.x[i], yi = in.y[i], zi = DIM == 3 ? in.z[i] : 0.0;
    const double rad = in.h[i] * in.radius_scale;
    const double rad2 = __dmul_rn(rad, rad);
    int cnt = 0;
    for (int dz = (DIM == 3 ? -1 : 0); dz <= (DIM == 3 ? 1 : 0); ++dz) {
        for (int dy = -1; dy <= 1; ++dy) {
            const int row = ((cz + dz) * H.n[1] + (cy + dy)) * H.n[0] + cx;
            const int b = v.start[row - 1], e = v.start[row + 2];
            if (b < 0 || e > in.n || b > e) {
                counts[i] = -1;
                return;
            }
            for (int k = b; k < e; ++k) {
                const int j = v.perm[k];
                const double dx = in.x[j] - xi;
                const double dy2 = in.y[j] - yi;
                const double dz2 = DIM == 3 ? in.z[j] - zi : 0.0;
                if (dist2_ref<DIM>(dx, dy2, dz2) < rad2) ++cnt;
            }
        }
    }
    counts[i] = cnt;
}

// Device address of sphb_static_scratch per device, looked up once.
static std::mutex g_mu;
static unsigned char *g_addr[256];

static int scratch_for_current_device(unsigned char **out)
{
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 256)
        return launch_status("sphb_neighbor_counts_static: cudaGetDevice");
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_addr[dev]) {
        void *p = nullptr;
        const cudaError_t err = cudaGetSymbolAddress(&p, sphb_static_scratch);
        if (err != cudaSuccess || !p)
            return launch_status("sphb_neighbor_counts_static: cudaGetSymbolAddress");
        g_addr[dev] = (unsigned char *)p;
    }
    *out = g_addr[dev];
    return SPHB_OK;
}

}  // namespace nalloc
}  // namespace sphb

using namespace sphb;
using namespace sphb::nalloc;

extern "C" int sphb_neighbor_counts_static(int32_t n, int32_t dim, const double *x,
                                           const double *y, const double *z,
                                           const double *h, double radius_scale,
                                           int32_t *counts, void *stream)
{
    if (n < 0 || n > SPHB_STATIC_MAX_PARTICLES) return SPHB_ERR_WORKSPACE;
    if (dim != 2 && dim != 3) return SPHB_ERR_UNSUPPORTED;
    if (!x || !y || !h || !counts || (dim == 3 && !z) || !(radius_scale > 0.0))
        return SPHB_ERR_ARG;
    if (n == 0) return SPHB_OK;
    unsigned char *base = nullptr;
    int rc = scratch_for_current_device(&base);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    Input in{n, dim, x, y, z, h, radius_scale};
    const int nb = (n + 255) / 256;
    k_reset<<<1, 32, 0, st>>>(base);
    k_bounds<<<nb, 256, 0, st>>>(base, in);
    k_grid<<<1, 1, 0, st>>>(base, in);
    k_zero<<<148, 256, 0, st>>>(base);   // one block per SM, grid-stride
    k_hash<<<nb, 256, 0, st>>>(base, in);
    k_scan<<<1, 1024, 0, st>>>(base);
    k_scatter<<<nb, 256, 0, st>>>(base, n);
    if (dim == 2) k_count<2><<<nb, 256, 0, st>>>(base, in, counts);
    else k_count<3><<<nb, 256, 0, st>>>(base, in, counts);
    return launch_status("sphb_neighbor_counts_static");
}
