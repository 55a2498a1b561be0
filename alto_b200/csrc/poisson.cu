// poisson.cu -- synthetic Poisson count tensors (cpd64 -d).
//
// Replaces PoissonGeneratorRun (IntelLabs/ALTO src/poisson_generator.cpp:
// 337-375) as called by MakeSparseTensor (src/main.cpp:652-675), following
// the same method step by step, with the reference's random streams:
//   GenerateRandomModel (:145-194)  host: every factor entry 0.1, then per
//       column ceil(0.2 I_n) entries (chosen by a partial Fisher-Yates
//       shuffle driven by the C library's rand()) set to uniform(1, 10R);
//       lambda uniform(0, 1); KruskalModelNormalize (1-norm columns into
//       lambda, kruskal_model.cpp:126-170); lambda scaled to sum 1.
//   GenerateEdges (:197-259)        device: multinomial component counts
//       (ProbCount: uniform draws binned on the cumulative lambda), then for
//       every component r and mode n its count of indices sampled from the
//       cumulative column U_n[:, r] (ProbSample, the same binary search,
//       Binning :37-56).
//   ConstructCIdx (:262-334)        device: sort by (i_{N-1}, ..., i_0) (the
//       reference's LSD counting sort by mode gives the same order) and
//       duplicates merged into counts.
// The reference draws its uniforms from one 64-bit Mersenne Twister per
// OpenMP thread (MT19937-64, M. Matsumoto and T. Nishimura, seeded 1234 +
// thread id; src/rng.cpp) and splits every batch of draws into contiguous
// equal chunks, one per thread (UniformRandom :21-34, batches of BSIZE =
// 100,000).  The generator here replays that schedule for a given thread
// count: the model's draws on the host, the edges' on the device, where one
// CTA advances each stream (the twist of 312 words in two dependent halves,
// then 312 tempered outputs in parallel) and a second kernel maps every
// draw back to its place in the reference's order.  For the same thread
// count the tensor and the model are the reference's bit for bit (the
// reference's own column sums are an OpenMP reduction whose order is not
// fixed above one thread; here partial sums are combined in thread order).
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "internal.cuh"

namespace altob {

namespace {

constexpr int MT_N = 312;
constexpr int MT_M = 156;
constexpr u64 MT_A = 0xB5026F5AA96619E9ULL;
constexpr u64 MT_UPPER = 0xFFFFFFFF80000000ULL;
constexpr u64 MT_LOWER = 0x000000007FFFFFFFULL;
constexpr u64 POIS_BSIZE = 100000;  // draws per batch (poisson_generator.cpp:13)
constexpr u64 POIS_SEED = 1234;     // stream t is seeded POIS_SEED + t (:14, :118)

struct MtState {
    u64 mt[MT_N];
    int mti;
};

__host__ __device__ __forceinline__ u64 mt_temper(u64 x)
{
    x ^= (x >> 29) & 0x5555555555555555ULL;
    x ^= (x << 17) & 0x71D67FFFEDA60000ULL;
    x ^= (x << 37) & 0xFFF7EEE000000000ULL;
    x ^= x >> 43;
    return x;
}

__host__ __device__ __forceinline__ u64 mt_mix(u64 a, u64 b, u64 c)
{
    const u64 x = (a & MT_UPPER) | (b & MT_LOWER);
    return c ^ (x >> 1) ^ ((x & 1ULL) ? MT_A : 0ULL);
}

// (x >> 12 + 0.5) / 2^52: the reference's uniform in (0, 1)
__host__ __device__ __forceinline__ double mt_unit(u64 x) { return ((double)(x >> 12) + 0.5) * (1.0 / 4503599627370496.0); }

void mt_seed(MtState& s, u64 seed)
{
    s.mt[0] = seed;
    for (int i = 1; i < MT_N; ++i) s.mt[i] = (u64)i + 6364136223846793005ULL * (s.mt[i - 1] ^ (s.mt[i - 1] >> 62));
    s.mti = MT_N;
}

void mt_twist(MtState& s)
{
    int i = 0;
    for (; i < MT_N - MT_M; ++i) s.mt[i] = mt_mix(s.mt[i], s.mt[i + 1], s.mt[i + MT_M]);
    for (; i < MT_N - 1; ++i) s.mt[i] = mt_mix(s.mt[i], s.mt[i + 1], s.mt[i + MT_M - MT_N]);
    s.mt[MT_N - 1] = mt_mix(s.mt[MT_N - 1], s.mt[0], s.mt[MT_M - 1]);
    s.mti = 0;
}

double mt_uniform(MtState& s)
{
    if (s.mti >= MT_N) mt_twist(s);
    return mt_unit(mt_temper(s.mt[s.mti++]));
}

// The reference's UniformRandom(n, low, high, a) on T streams: thread t
// fills a[t*chunk, min((t+1)*chunk, n)) from its own stream.
void host_uniform(std::vector<MtState>& st, u64 n, double low, double high, double* a)
{
    const u64 T = st.size();
    const u64 chunk = (n + T - 1) / T;
    for (u64 t = 0; t < T; ++t) {
        const u64 b = t * chunk, e = std::min(b + chunk, n);
        for (u64 i = b; i < e; ++i) a[i] = mt_uniform(st[t]) * (high - low) + low;
    }
}

// Binning (poisson_generator.cpp:37-56): the bin of rv in the cumulative
// table bins[0..nbins-1]; an exact hit on the last edge is the last bin.
__host__ __device__ __forceinline__ u64 pois_bin(double rv, u64 nbins, const double* bins)
{
    long long start = 0, end = (long long)nbins - 1;
    while (start <= end) {
        const long long mid = (end + start) / 2;
        if (rv > bins[mid]) {
            start = mid + 1;
        } else if (rv == bins[mid]) {
            return (u64)(mid == (long long)nbins - 1 ? mid - 1 : mid);
        } else {
            end = mid - 1;
        }
    }
    return (u64)end;
}

// One UniformRandom call of the edge phase: `len` draws starting at global
// draw `g0`, split over the streams in chunks of `chunk`; the draws of
// stream t start at position sstart[call * T + t] of that stream's sequence.
struct PoisCall {
    u64 g0, len, chunk;
    u64 bins_off, nbins;  // cumulative table of the call
    u64 dst;              // ProbSample: first edge written; ProbCount: unused
    int mode;             // ProbSample: mode written; -1: ProbCount
};

// One CTA per stream: advances MT19937-64 from its saved state and writes
// `len[t]` uniforms to out + off[t] in stream order.
__global__ void __launch_bounds__(320) k_mt_run(MtState* __restrict__ states, const u64* __restrict__ off,
                                                const u64* __restrict__ len, double* __restrict__ out)
{
    __shared__ u64 s[MT_N];
    const int t = blockIdx.x, tid = threadIdx.x;
    MtState* g = states + t;
    for (int i = tid; i < MT_N; i += blockDim.x) s[i] = g->mt[i];
    int mti = g->mti;
    __syncthreads();
    const u64 n = len[t];
    double* o = out + off[t];
    u64 done = 0;
    while (done < n) {
        if (mti >= MT_N) {
            // twist: words 0..155 from the old state, then 156..311 from the
            // old state and the new words 0..155
            u64 a = 0, b = 0, c = 0;
            if (tid < MT_N) {
                a = s[tid];
                b = tid + 1 < MT_N ? s[tid + 1] : 0;
                c = tid < MT_N - MT_M ? s[tid + MT_M] : 0;
            }
            __syncthreads();
            if (tid < MT_N - MT_M) s[tid] = mt_mix(a, b, c);
            __syncthreads();
            if (tid >= MT_N - MT_M && tid < MT_N - 1) s[tid] = mt_mix(a, b, s[tid - (MT_N - MT_M)]);
            if (tid == MT_N - 1) s[tid] = mt_mix(a, s[0], s[MT_M - 1]);
            __syncthreads();
            mti = 0;
        }
        const u64 avail = min((u64)(MT_N - mti), n - done);
        for (u64 j = tid; j < avail; j += blockDim.x) o[done + j] = mt_unit(mt_temper(s[mti + j]));
        done += avail;
        mti += (int)avail;
        __syncthreads();
    }
    for (int i = tid; i < MT_N; i += blockDim.x) g->mt[i] = s[i];
    if (tid == 0) g->mti = mti;
}

// Every draw of the phase binned at its place in the reference's order.
__global__ void k_pois_bin(const PoisCall* __restrict__ calls, int ncalls, u64 total, const u64* __restrict__ sstart,
                           int T, const double* __restrict__ seq, const u64* __restrict__ seq_off,
                           const double* __restrict__ bins, int nmode, unsigned long long* __restrict__ counts,
                           u32* __restrict__ eidx)
{
    for (u64 g = (u64)blockIdx.x * blockDim.x + threadIdx.x; g < total; g += (u64)gridDim.x * blockDim.x) {
        int lo = 0, hi = ncalls - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (calls[mid].g0 <= g) lo = mid;
            else hi = mid - 1;
        }
        const PoisCall c = calls[lo];
        const u64 i = g - c.g0;
        const u64 t = i / c.chunk;
        const double rv = seq[seq_off[t] + sstart[(u64)lo * T + t] + (i - t * c.chunk)];
        const u64 b = pois_bin(rv, c.nbins, bins + c.bins_off);
        if (c.mode < 0) atomicAdd(counts + b, 1ull);
        else eidx[(c.dst + i) * (u64)nmode + c.mode] = (u32)b;
    }
}

// Coordinates -> one sort key, mode N-1 most significant (the order of the
// reference's LSD counting sort by mode 0, 1, ..., N-1).
__global__ void k_pois_keys(const u32* __restrict__ eidx, u64 n, int nmode, const int* __restrict__ shift, int kw,
                            u64* __restrict__ klo, u64* __restrict__ khi, u32* __restrict__ iota)
{
    for (u64 e = (u64)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (u64)gridDim.x * blockDim.x) {
        u64 lo = 0, hi = 0;
        for (int m = 0; m < nmode; ++m) {
            const u64 v = eidx[e * nmode + m];
            const int s = shift[m];
            if (s < 64) {
                lo |= v << s;
                if (s > 0 && s + 32 > 64) hi |= v >> (64 - s);
            } else {
                hi |= v << (s - 64);
            }
        }
        klo[e] = lo;
        if (kw == 2) khi[e] = hi;
        iota[e] = (u32)e;
    }
}

__global__ void k_pois_heads(const u64* __restrict__ klo, const u64* __restrict__ khi, u64 n, u32* __restrict__ head)
{
    for (u64 e = (u64)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (u64)gridDim.x * blockDim.x)
        head[e] = e == 0 || klo[e] != klo[e - 1] || (khi && khi[e] != khi[e - 1]);
}

// Distinct coordinates and their counts: position k of the output gets the
// k-th run of equal keys (start found by the head flags' running count).
__global__ void k_pois_emit(const u32* __restrict__ head, const u64* __restrict__ rank_incl, const u32* __restrict__ perm,
                            const u32* __restrict__ eidx, u64 n, int nmode, u64* __restrict__ start)
{
    for (u64 e = (u64)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (u64)gridDim.x * blockDim.x)
        if (head[e]) start[rank_incl[e] - 1] = e;
}

__global__ void k_pois_out(const u64* __restrict__ start, u64 nnz, u64 n, const u32* __restrict__ perm,
                           const u32* __restrict__ eidx, int nmode, u64* __restrict__ cidx, double* __restrict__ vals)
{
    for (u64 k = (u64)blockIdx.x * blockDim.x + threadIdx.x; k < nnz; k += (u64)gridDim.x * blockDim.x) {
        const u64 s = start[k], e = k + 1 < nnz ? start[k + 1] : n;
        const u32 p = perm[s];
        for (int m = 0; m < nmode; ++m) cidx[(u64)m * nnz + k] = eidx[(u64)p * nmode + m];
        vals[k] = (double)(e - s);
    }
}

__global__ void k_u32_to_u64(const u32* __restrict__ a, u64 n, u64* __restrict__ b)
{
    for (u64 e = (u64)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (u64)gridDim.x * blockDim.x) b[e] = a[e];
}

// Inclusive running sum of u64 values (one CTA per 1024-element block, then
// the block totals): the run ranks of the head flags.
__global__ void k_scan_blocks(const u64* __restrict__ in, u64 n, u64* __restrict__ out, u64* __restrict__ totals)
{
    __shared__ u64 sh[1024];
    const u64 i = (u64)blockIdx.x * 1024 + threadIdx.x;
    u64 v = i < n ? in[i] : 0;
    sh[threadIdx.x] = v;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
        const u64 add = threadIdx.x >= (unsigned)o ? sh[threadIdx.x - o] : 0;
        __syncthreads();
        sh[threadIdx.x] += add;
        __syncthreads();
    }
    if (i < n) out[i] = sh[threadIdx.x];
    if (threadIdx.x == 1023) totals[blockIdx.x] = sh[1023];
}

__global__ void k_scan_add(u64* __restrict__ out, u64 n, const u64* __restrict__ base)
{
    const u64 i = (u64)blockIdx.x * 1024 + threadIdx.x;
    if (i < n && blockIdx.x > 0) out[i] += base[blockIdx.x - 1];
}

static int pgrid(u64 n) { return (int)std::max<u64>(1, std::min<u64>((n + 255) / 256, (u64)num_sms() * 16)); }

// Inclusive scan of n u64 values (recursive over the block totals).
static altob_status scan_u64(u64* d, u64 n, cudaStream_t st)
{
    if (n == 0) return ALTOB_OK;
    const u64 nb = (n + 1023) / 1024;
    u64* tot = nullptr;
    ALTOB_TRY(dmalloc_t(&tot, nb));
    k_scan_blocks<<<(unsigned)nb, 1024, 0, st>>>(d, n, d, tot);
    altob_status s = cudaGetLastError() == cudaSuccess ? ALTOB_OK : fail(ALTOB_ERR_CUDA, "scan launch failed");
    if (s == ALTOB_OK && nb > 1) s = scan_u64(tot, nb, st);
    if (s == ALTOB_OK && nb > 1) k_scan_add<<<(unsigned)nb, 1024, 0, st>>>(d, n, tot);
    dfree(tot);
    return s;
}

// Device-side uniforms of one phase: every stream's part of every call.
struct Phase {
    std::vector<PoisCall> calls;
    std::vector<u64> sstart;  // ncalls x T
    std::vector<u64> per;     // draws per stream
    u64 total = 0;
    int T = 1;
    explicit Phase(int t) : per(t, 0), T(t) {}
    void add(u64 len, u64 bins_off, u64 nbins, u64 dst, int mode)
    {
        for (u64 b = 0; b < len; b += POIS_BSIZE) {
            const u64 l = std::min(POIS_BSIZE, len - b);
            const u64 chunk = (l + T - 1) / T;
            PoisCall c{total, l, chunk, bins_off, nbins, dst + b, mode};
            for (int t = 0; t < T; ++t) {
                const u64 s0 = (u64)t * chunk, s1 = std::min(s0 + chunk, l);
                sstart.push_back(per[t]);
                per[t] += s1 > s0 ? s1 - s0 : 0;
            }
            calls.push_back(c);
            total += l;
        }
    }
};

struct DevBuf {
    std::vector<void*> p;
    ~DevBuf()
    {
        for (void* x : p) dfree(x);
    }
    template <typename T>
    altob_status get(T** out, u64 n)
    {
        ALTOB_TRY(dmalloc_t(out, n));
        p.push_back(*out);
        return ALTOB_OK;
    }
};

// Runs a phase: streams advanced on the device, every draw binned.
static altob_status run_phase(const Phase& ph, MtState* d_states, const double* d_bins, int nmode,
                              unsigned long long* d_counts, u32* d_eidx, cudaStream_t st)
{
    if (ph.total == 0) return ALTOB_OK;
    DevBuf buf;
    const int T = ph.T;
    std::vector<u64> off(T, 0);
    u64 all = 0;
    for (int t = 0; t < T; ++t) {
        off[t] = all;
        all += ph.per[t];
    }
    double* seq = nullptr;
    u64 *d_off = nullptr, *d_len = nullptr, *d_ss = nullptr;
    PoisCall* d_calls = nullptr;
    ALTOB_TRY(buf.get(&seq, all));
    ALTOB_TRY(buf.get(&d_off, T));
    ALTOB_TRY(buf.get(&d_len, T));
    ALTOB_TRY(buf.get(&d_ss, ph.sstart.size()));
    ALTOB_TRY(buf.get(&d_calls, ph.calls.size()));
    ALTOB_CUDA(cudaMemcpyAsync(d_off, off.data(), T * 8, cudaMemcpyHostToDevice, st));
    ALTOB_CUDA(cudaMemcpyAsync(d_len, ph.per.data(), T * 8, cudaMemcpyHostToDevice, st));
    ALTOB_CUDA(cudaMemcpyAsync(d_ss, ph.sstart.data(), ph.sstart.size() * 8, cudaMemcpyHostToDevice, st));
    ALTOB_CUDA(cudaMemcpyAsync(d_calls, ph.calls.data(), ph.calls.size() * sizeof(PoisCall), cudaMemcpyHostToDevice,
                               st));
    k_mt_run<<<T, 320, 0, st>>>(d_states, d_off, d_len, seq);
    ALTOB_LAUNCH_CHECK();
    k_pois_bin<<<pgrid(ph.total), 256, 0, st>>>(d_calls, (int)ph.calls.size(), ph.total, d_ss, T, seq, d_off, d_bins,
                                                nmode, d_counts, d_eidx);
    ALTOB_LAUNCH_CHECK();
    ALTOB_CUDA(cudaStreamSynchronize(st));  // the host vectors go out of scope
    return ALTOB_OK;
}

}  // namespace

// The whole generator; see the file comment.  U / lam (host, FP64) receive
// the model; *out the tensor (host COO, 0-based, values = counts).
static altob_status poisson_impl(int nmode, const u64* dims, u64 num_edges, u64 R, int T, double* const* U_out,
                                 double* lam_out, altob_coo** out, cudaStream_t st)
{
    u64 maxd = 0;
    for (int n = 0; n < nmode; ++n) maxd = std::max(maxd, dims[n]);
    std::vector<MtState> ms(T);
    for (int t = 0; t < T; ++t) mt_seed(ms[t], POIS_SEED + (u64)t);
    // the C library's rand() from its initial state (the reference never
    // seeds it before generating), through a private glibc random_r state
    char rstate[128];
    random_data rd;
    memset(&rd, 0, sizeof(rd));
    memset(rstate, 0, sizeof(rstate));
    if (initstate_r(1, rstate, sizeof(rstate), &rd) != 0) return fail(ALTOB_ERR_CUDA, "initstate_r failed");
    auto crand = [&]() {
        int32_t r = 0;
        random_r(&rd, &r);
        return (u64)r;
    };
    // ---- GenerateRandomModel
    std::vector<std::vector<double>> U(nmode);
    std::vector<u64> perm(maxd + 1);
    std::vector<double> vals(maxd + 1);
    for (int n = 0; n < nmode; ++n) {
        const u64 dn = dims[n];
        U[n].assign(dn * R, 0.1);
        const u64 nbig = (u64)std::ceil(0.2 * (double)dn);
        for (u64 r = 0; r < R; ++r) {
            for (u64 i = 0; i < dn; ++i) perm[i] = i;
            for (u64 i = 0; i < nbig; ++i) {
                const u64 idx = crand() % (dn - i) + i;
                std::swap(perm[i], perm[idx]);
            }
            host_uniform(ms, nbig, 1.0, 10.0 * (double)R, vals.data());
            for (u64 i = 0; i < nbig; ++i) U[n][perm[i] * R + r] = vals[i];
        }
    }
    std::vector<double> lam(R, 0.0);
    host_uniform(ms, R, 0.0, 1.0, lam.data());
    // KruskalModelNormalize: per mode, column 1-norms summed over the rows
    // of each thread's share of an OpenMP static schedule (n / T rows, one
    // more for the first n % T threads), the partial sums combined in thread
    // order, columns divided, norms absorbed into lambda
    for (int n = 0; n < nmode; ++n) {
        const u64 dn = dims[n];
        std::vector<double> cn(R, 0.0);
        const u64 q = dn / (u64)T, extra = dn % (u64)T;
        for (int t = 0; t < T; ++t) {
            std::vector<double> part(R, 0.0);
            const u64 b = (u64)t * q + std::min<u64>((u64)t, extra);
            const u64 e = b + q + ((u64)t < extra ? 1 : 0);
            for (u64 i = b; i < e; ++i)
                for (u64 j = 0; j < R; ++j) part[j] += std::fabs(U[n][i * R + j]);
            for (u64 j = 0; j < R; ++j) cn[j] += part[j];
        }
        for (u64 i = 0; i < dn; ++i)
            for (u64 j = 0; j < R; ++j) U[n][i * R + j] /= cn[j];
        for (u64 j = 0; j < R; ++j) lam[j] *= cn[j];
    }
    double tmp = 0.0;
    for (u64 j = 0; j < R; ++j) tmp += lam[j];
    if (tmp == 0.0) return fail(ALTOB_ERR_ARG, "Poisson generator: lambda sums to 0");
    tmp = 1.0 / tmp;
    for (u64 j = 0; j < R; ++j) lam[j] *= tmp;

    // ---- GenerateEdges: cumulative tables (lambda, then every column)
    std::vector<double> bins;
    bins.push_back(0.0);
    for (u64 i = 0; i < R; ++i) bins.push_back(std::min(lam[i] + bins[i], 1.0));
    std::vector<u64> col_off((size_t)nmode * R);
    for (int n = 0; n < nmode; ++n)
        for (u64 r = 0; r < R; ++r) {
            const u64 o = bins.size();
            col_off[(size_t)n * R + r] = o;
            bins.push_back(0.0);
            for (u64 i = 0; i < dims[n]; ++i) bins.push_back(std::min(U[n][i * R + r] + bins[o + i], 1.0));
        }
    DevBuf buf;
    MtState* d_states = nullptr;
    double* d_bins = nullptr;
    unsigned long long* d_counts = nullptr;
    ALTOB_TRY(buf.get(&d_states, T));
    ALTOB_TRY(buf.get(&d_bins, bins.size()));
    ALTOB_TRY(buf.get(&d_counts, R + 2));
    ALTOB_CUDA(cudaMemcpyAsync(d_states, ms.data(), T * sizeof(MtState), cudaMemcpyHostToDevice, st));
    ALTOB_CUDA(cudaMemcpyAsync(d_bins, bins.data(), bins.size() * 8, cudaMemcpyHostToDevice, st));
    ALTOB_CUDA(cudaMemsetAsync(d_counts, 0, (R + 2) * 8, st));
    // ProbCount: component counts
    {
        Phase pc(T);
        pc.add(num_edges, 0, R + 1, 0, -1);
        ALTOB_TRY(run_phase(pc, d_states, d_bins, nmode, d_counts, nullptr, st));
    }
    std::vector<unsigned long long> rc(R + 2, 0);
    ALTOB_CUDA(cudaMemcpyAsync(rc.data(), d_counts, (R + 2) * 8, cudaMemcpyDeviceToHost, st));
    ALTOB_CUDA(cudaStreamSynchronize(st));
    // ProbSample: for every component, every mode's indices (draws that fell
    // past the last component edge, bin R, are not sampled)
    u64 edges = 0;
    Phase ps(T);
    for (u64 r = 0; r < R; ++r) {
        for (int n = 0; n < nmode; ++n) ps.add(rc[r], col_off[(size_t)n * R + r], dims[n] + 1, edges, n);
        edges += rc[r];
    }
    u32* d_eidx = nullptr;
    ALTOB_TRY(buf.get(&d_eidx, std::max<u64>(1, edges * nmode)));
    ALTOB_TRY(run_phase(ps, d_states, d_bins, nmode, d_counts, d_eidx, st));
    // lambda rescaled to the number of edges asked for (:254-256)
    for (u64 r = 0; r < R; ++r) lam[r] *= (double)num_edges;

    // ---- ConstructCIdx: sort, merge duplicates
    int shift[ALTOB_MAX_MODES], bits = 0;
    for (int n = 0; n < nmode; ++n) {
        shift[n] = bits;
        int b = 0;
        while (b < 32 && (1ull << b) < dims[n] + 1) ++b;  // + 1: a bin past the end stays distinct
        bits += b;
    }
    if (bits > 128) return fail(ALTOB_ERR_UNSUPPORTED, "Poisson generator: coordinates need more than 128 bits");
    const int kw = bits > 64 ? 2 : 1;
    u64 *klo = nullptr, *khi = nullptr, *klo2 = nullptr, *khi2 = nullptr, *start = nullptr, *rank_incl = nullptr;
    u32 *iota = nullptr, *iota2 = nullptr, *head = nullptr;
    int* d_shift = nullptr;
    const u64 E = std::max<u64>(1, edges);
    ALTOB_TRY(buf.get(&klo, E));
    ALTOB_TRY(buf.get(&klo2, E));
    if (kw == 2) {
        ALTOB_TRY(buf.get(&khi, E));
        ALTOB_TRY(buf.get(&khi2, E));
    }
    ALTOB_TRY(buf.get(&iota, E));
    ALTOB_TRY(buf.get(&iota2, E));
    ALTOB_TRY(buf.get(&head, E));
    ALTOB_TRY(buf.get(&rank_incl, E));
    ALTOB_TRY(buf.get(&start, E));
    ALTOB_TRY(buf.get(&d_shift, ALTOB_MAX_MODES));
    ALTOB_CUDA(cudaMemcpyAsync(d_shift, shift, sizeof(shift), cudaMemcpyHostToDevice, st));
    u64 nnz = 0;
    if (edges) {
        k_pois_keys<<<pgrid(edges), 256, 0, st>>>(d_eidx, edges, nmode, d_shift, kw, klo, khi, iota);
        ALTOB_LAUNCH_CHECK();
        bool alt = false;
        ALTOB_TRY(radix_sort_pairs(klo, khi, iota, klo2, khi2, iota2, edges, kw, bits, st, &alt));
        const u64* sk = alt ? klo2 : klo;
        const u64* sh = kw == 2 ? (alt ? khi2 : khi) : nullptr;
        const u32* sp = alt ? iota2 : iota;
        k_pois_heads<<<pgrid(edges), 256, 0, st>>>(sk, sh, edges, head);
        ALTOB_LAUNCH_CHECK();
        k_u32_to_u64<<<pgrid(edges), 256, 0, st>>>(head, edges, rank_incl);
        ALTOB_LAUNCH_CHECK();
        ALTOB_TRY(scan_u64(rank_incl, edges, st));
        ALTOB_CUDA(cudaMemcpyAsync(&nnz, rank_incl + edges - 1, 8, cudaMemcpyDeviceToHost, st));
        k_pois_emit<<<pgrid(edges), 256, 0, st>>>(head, rank_incl, sp, d_eidx, edges, nmode, start);
        ALTOB_LAUNCH_CHECK();
        ALTOB_CUDA(cudaStreamSynchronize(st));
        u64* d_cidx = nullptr;
        double* d_vals = nullptr;
        ALTOB_TRY(buf.get(&d_cidx, std::max<u64>(1, nnz * nmode)));
        ALTOB_TRY(buf.get(&d_vals, std::max<u64>(1, nnz)));
        k_pois_out<<<pgrid(nnz), 256, 0, st>>>(start, nnz, edges, sp, d_eidx, nmode, d_cidx, d_vals);
        ALTOB_LAUNCH_CHECK();
        altob_coo* c = (altob_coo*)calloc(1, sizeof(altob_coo));
        if (!c) return fail(ALTOB_ERR_NOMEM, "host allocation");
        c->nmode = nmode;
        c->nnz = nnz;
        for (int n = 0; n < nmode; ++n) c->dims[n] = dims[n];
        c->cidx = (uint64_t*)malloc(std::max<u64>(1, nnz * nmode) * 8);
        c->vals = (double*)malloc(std::max<u64>(1, nnz) * 8);
        if (!c->cidx || !c->vals) {
            altob_coo_free(c);
            return fail(ALTOB_ERR_NOMEM, "host allocation");
        }
        cudaMemcpyAsync(c->cidx, d_cidx, nnz * nmode * 8, cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(c->vals, d_vals, nnz * 8, cudaMemcpyDeviceToHost, st);
        const cudaError_t e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) {
            altob_coo_free(c);
            return fail(ALTOB_ERR_CUDA, std::string("Poisson generator: ") + cudaGetErrorString(e));
        }
        *out = c;
    } else {
        altob_coo* c = (altob_coo*)calloc(1, sizeof(altob_coo));
        if (!c) return fail(ALTOB_ERR_NOMEM, "host allocation");
        c->nmode = nmode;
        for (int n = 0; n < nmode; ++n) c->dims[n] = dims[n];
        c->cidx = (uint64_t*)malloc(8);
        c->vals = (double*)malloc(8);
        *out = c;
    }
    for (int n = 0; n < nmode && U_out; ++n)
        if (U_out[n]) memcpy(U_out[n], U[n].data(), U[n].size() * 8);
    if (lam_out) memcpy(lam_out, lam.data(), R * 8);
    return ALTOB_OK;
}

}  // namespace altob

using namespace altob;

extern "C" altob_status altob_poisson_tensor(int nmode, const uint64_t* dims, uint64_t num_edges, uint64_t rank,
                                             int nthreads, double* const* model_U, double* model_lambda,
                                             altob_coo** out, void* stream)
{
    if (!dims || !out) return fail(ALTOB_ERR_ARG, "NULL argument");
    *out = nullptr;
    if (nmode < 1 || nmode > ALTOB_MAX_MODES) return fail(ALTOB_ERR_ARG, "nmode must be 1..5");
    if (rank < 1) return fail(ALTOB_ERR_ARG, "rank must be >= 1");
    if (nthreads < 1 || nthreads > 4096) return fail(ALTOB_ERR_ARG, "nthreads must be 1..4096");
    if (num_edges == 0) return fail(ALTOB_ERR_ARG, "num_edges must be > 0 (the reference asserts it)");
    if (num_edges >= (1ull << 32)) return fail(ALTOB_ERR_UNSUPPORTED, "num_edges must be below 2^32");
    for (int n = 0; n < nmode; ++n) {
        if (dims[n] < rank) return fail(ALTOB_ERR_ARG, "every dimension must be >= rank (the reference asserts it)");
        if (dims[n] >= (1ull << 31)) return fail(ALTOB_ERR_UNSUPPORTED, "dimensions must be below 2^31");
    }
    cudaStream_t st = (cudaStream_t)stream;
    StreamScope scope(st);
    return poisson_impl(nmode, dims, num_edges, rank, nthreads, model_U, model_lambda, out, st);
}
