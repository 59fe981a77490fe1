// Density-matrix simulation, as the reference's noise variant does it
// (svsim_qsharp_noise/svsim_nvgpu_sin.cuh: rho of n qubits held as a vector of 2n qubits,
// dim = 2^(2n) at :527-529, every noisy gate a superoperator on the row and column
// copies of its qubits).
//
// rho[i][j] sits at index i + 2^n j, so qubit q of the row index is vector qubit q and
// qubit q of the column index is vector qubit q + n.  A unitary U acts as
// rho -> U rho U^dagger = (U on the row qubits) (conj U on the column qubits).  Each
// elementary op of a gate's lowering becomes
//   * a one-qubit matrix M: one 4x4 block M (x) conj(M) on the pair (q, q + n);
//   * CX(c, t): CX on (c, t) and CX on (c + n, t + n) (real, its own conjugate);
// and a one-qubit channel with Kraus operators K_k becomes the block sum_k K_k (x) conj(K_k)
// on (q, q + n), applied after every gate to each qubit the gate touches.  The blocks are
// F_M4 ops: the pair engine (FP64 tensor cores) takes them as two-qubit blocks; below its
// 12-qubit tile the per-gate engine applies them with k_m4.
#include <algorithm>
#include <cmath>
#include <complex>
#include <string>

#include "gate_math.cuh"

namespace svb {
namespace {

template <typename T>
__global__ void __launch_bounds__(256)
k_m4(typename VecOf<T>::type* __restrict__ sv, uint64_t quads, int q0, int q1, Coef<T> lo, Coef<T> hi,
     Coef<T> lo2, Coef<T> hi2)
{
    // the 4x4 matrix: rows 0..1 in lo, hi (8 coefficients each: 4 complex), rows 2..3 in lo2, hi2
    using V = typename VecOf<T>::type;
    const int a = q0 < q1 ? q0 : q1, b = q0 < q1 ? q1 : q0;
    const uint64_t d0 = 1ull << q0, d1 = 1ull << q1;
    const T* rows[4] = {lo.m, hi.m, lo2.m, hi2.m};
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < quads;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t base = insert_zero(insert_zero(i, a), b);
        const uint64_t idx[4] = {base, base | d0, base | d1, base | d0 | d1};
        V x[4];
#pragma unroll
        for (int k = 0; k < 4; k++) x[k] = sv[idx[k]];
#pragma unroll
        for (int r = 0; r < 4; r++) {
            T re = 0, im = 0;
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const T mr = rows[r][2 * k], mi = rows[r][2 * k + 1];
                re += mr * x[k].x - mi * x[k].y;
                im += mr * x[k].y + mi * x[k].x;
            }
            V y;
            y.x = re;
            y.y = im;
            sv[idx[r]] = y;
        }
    }
}

// p[i] = Re rho[i][i] = Re vec[i + 2^n i]
template <typename T>
__global__ void k_dm_diag(const typename VecOf<T>::type* __restrict__ sv, uint64_t dim, int n, double* __restrict__ p)
{
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < dim;
         i += (uint64_t)gridDim.x * blockDim.x)
        p[i] = (double)sv[i + (i << n)].x;
}

using cplx = std::complex<double>;

// 2x2 matrix of an elementary op (read off the kernels' expressions on the basis)
void matrix2(const EOp& e, cplx u[4])
{
    const Coef<double> c = load_coef<double>(e.m);
    for (int col = 0; col < 2; col++) {
        double2 a0 = make_double2(col == 0 ? 1.0 : 0.0, 0.0), a1 = make_double2(col == 1 ? 1.0 : 0.0, 0.0);
        if (form_is_diag(e.form)) {
            diag_one<double>(e.form, c, a1);
            if (e.form == F_DIAG) diag_zero<double>(e.form, c, a0);
        } else {
            dense_pair<double>(e.form, c, a0, a1);
        }
        u[col] = cplx(a0.x, a0.y);
        u[2 + col] = cplx(a1.x, a1.y);
    }
}

// the superoperator sum_k K_k (x) conj(K_k) (K_k on bit 0, conj K_k on bit 1)
Mat4 superop(const cplx* kraus, int nk)
{
    cplx s[16] = {};
    for (int k = 0; k < nk; k++) {
        const cplx* K = kraus + 4 * k;
        for (int ap = 0; ap < 4; ap++)
            for (int a = 0; a < 4; a++)
                s[ap * 4 + a] += K[(ap & 1) * 2 + (a & 1)] * std::conj(K[(ap >> 1) * 2 + (a >> 1)]);
    }
    Mat4 m;
    for (int i = 0; i < 16; i++) {
        m[2 * i] = s[i].real();
        m[2 * i + 1] = s[i].imag();
    }
    return m;
}

}  // namespace

template <typename T>
cudaError_t launch_m4(void* state, int n, int q0, int q1, const Mat4& m, cudaStream_t s)
{
    using V = typename VecOf<T>::type;
    Coef<T> r[4];
    for (int row = 0; row < 4; row++)
        for (int k = 0; k < 8; k++) r[row].m[k] = static_cast<T>(m[row * 8 + k]);
    const uint64_t quads = 1ull << (n - 2);
    const unsigned grid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((quads + 255) / 256, 148ull * 8));
    k_m4<T><<<grid, 256, 0, s>>>(static_cast<V*>(state), quads, q0, q1, r[0], r[1], r[2], r[3]);
    return cudaGetLastError();
}
template cudaError_t launch_m4<double>(void*, int, int, int, const Mat4&, cudaStream_t);
template cudaError_t launch_m4<float>(void*, int, int, int, const Mat4&, cudaStream_t);

}  // namespace svb

using namespace svb;

extern "C" {

svb_status svb_dm_create(uint32_t n_qubits, int device, svb_sim** out)
{
    if (!out) { set_error("svb_dm_create: out is NULL"); return SVB_ERR_INVALID; }
    *out = nullptr;
    if (n_qubits < 1 || n_qubits > 17) {
        set_error("svb_dm_create: n_qubits must be in [1, 17] (the state holds 2 n qubits)");
        return SVB_ERR_INVALID;
    }
    svb_status st = svb_create(2 * n_qubits, device, SVB_FP64, out);
    if (st != SVB_OK) return st;
    (*out)->dm_qubits = n_qubits;
    return SVB_OK;
}

svb_status svb_dm_set_circuit(svb_sim* s, const svb_gate* gates, size_t n_gates, const double* noise_kraus,
                              uint32_t n_kraus)
{
    return svb_dm_set_circuit_superops(s, gates, n_gates, noise_kraus, n_kraus, nullptr, 0);
}

svb_status svb_dm_set_circuit_superops(svb_sim* s, const svb_gate* gates, size_t n_gates,
                                       const double* noise_kraus, uint32_t n_kraus,
                                       const svb_superop* superops, size_t n_superops)
{
    if (!s || (n_gates && !gates) || (n_kraus && !noise_kraus) || (n_superops && !superops)) {
        set_error("svb_dm_set_circuit: NULL argument");
        return SVB_ERR_INVALID;
    }
    // per-op superoperator tables: the reference's order (r = 2 i + j for rho[i][j] on the
    // gate's qubit) permuted into the F_M4 order of the pair (q, q + n) (a = i + 2 j)
    std::vector<int> table_of(64, -1);
    std::vector<Mat4> tables;
    for (size_t t = 0; t < n_superops; t++) {
        const uint32_t op = superops[t].op;
        if (op >= 64 || gate_qubit_slots(op) != 1) {
            set_error("svb_dm_set_circuit: superoperator " + std::to_string(t) + " is not for a one-qubit op");
            return SVB_ERR_INVALID;
        }
        static const int sigma[4] = {0, 2, 1, 3};
        Mat4 m;
        for (int a = 0; a < 4; a++)
            for (int b = 0; b < 4; b++) {
                m[(a * 4 + b) * 2] = superops[t].m[(sigma[a] * 4 + sigma[b]) * 2];
                m[(a * 4 + b) * 2 + 1] = superops[t].m[(sigma[a] * 4 + sigma[b]) * 2 + 1];
            }
        table_of[op] = (int)tables.size();
        tables.push_back(m);
    }
    if (!s->dm_qubits) { set_error("svb_dm_set_circuit: not a density-matrix handle (svb_dm_create)"); return SVB_ERR_STATE; }
    if (n_kraus > 16) { set_error("svb_dm_set_circuit: at most 16 Kraus operators"); return SVB_ERR_INVALID; }
    const uint32_t n = s->dm_qubits;
    // lower with the row qubits, then write the superoperator circuit on 2n qubits
    std::vector<EOp> eops;
    for (size_t i = 0; i < n_gates; i++) {
        const svb_gate& g = gates[i];
        const int slots = gate_qubit_slots(g.op);
        if (slots == 0) { set_error("svb_dm_set_circuit: gate " + std::to_string(i) + ": unknown op"); return SVB_ERR_INVALID; }
        for (int k = 0; k < slots; k++) {
            if (g.qb[k] >= n) {
                set_error("svb_dm_set_circuit: gate " + std::to_string(i) + " acts on a qubit >= n_qubits");
                return SVB_ERR_INVALID;
            }
            for (int j = 0; j < k; j++)
                if (g.qb[j] == g.qb[k]) {
                    set_error("svb_dm_set_circuit: gate " + std::to_string(i) + " repeats a qubit");
                    return SVB_ERR_INVALID;
                }
        }
        if (g.op < 64 && table_of[g.op] >= 0) {
            // the gate's own superoperator (noise included, as the reference's noisy gates)
            EOp b;
            b.form = F_M4;
            b.q = g.qb[0];
            b.c = g.qb[0] + n;
            b.mat = -2 - table_of[g.op];          // resolved below
            b.gate = (int32_t)i;
            eops.push_back(b);
            continue;
        }
        const size_t first = eops.size();
        if (!lower_gate(g, (int32_t)i, eops)) {
            set_error("svb_dm_set_circuit: gate " + std::to_string(i) + ": unknown op");
            return SVB_ERR_INVALID;
        }
        for (size_t k = first; k < eops.size(); k++)
            if (eops[k].form == F_SRN) {
                set_error("svb_dm_set_circuit: SRN is not complex-linear and has no superoperator");
                return SVB_ERR_UNSUPPORTED;
            }
        // mark where each gate ends, with the qubits it touched (for the noise blocks)
        EOp mark;
        mark.form = F_COUNT;
        mark.gate = (int32_t)i;
        uint32_t touched = 0;
        for (int k = 0; k < slots; k++) touched |= 1u << g.qb[k];
        mark.q = touched;
        eops.push_back(mark);
    }
    std::vector<cplx> kraus(4 * (size_t)n_kraus);
    for (uint32_t k = 0; k < 4 * n_kraus; k++) kraus[k] = cplx(noise_kraus[2 * k], noise_kraus[2 * k + 1]);
    std::vector<EOp> dm;
    std::vector<Mat4> mats;
    int noise_mat = -1;
    if (n_kraus) {
        noise_mat = (int)mats.size();
        mats.push_back(superop(kraus.data(), (int)n_kraus));
    }
    const int table_base = (int)mats.size();
    mats.insert(mats.end(), tables.begin(), tables.end());
    for (const EOp& e : eops) {
        if (e.form == F_M4 && e.mat <= -2) {
            EOp b = e;
            b.mat = table_base + (-2 - e.mat);
            dm.push_back(b);
            continue;
        }
        if (e.form == F_COUNT) {
            if (noise_mat < 0) continue;
            for (uint32_t q = 0; q < n; q++)
                if ((e.q >> q) & 1u) {
                    EOp b;
                    b.form = F_M4;
                    b.q = q;
                    b.c = q + n;
                    b.mat = noise_mat;
                    b.gate = e.gate;
                    dm.push_back(b);
                }
            continue;
        }
        if (e.form == F_CX) {
            dm.push_back(e);
            EOp c2 = e;
            c2.q += n;
            c2.c += n;
            dm.push_back(c2);
            continue;
        }
        cplx u[4];
        matrix2(e, u);
        cplx uu[4] = {u[0], u[1], u[2], u[3]};
        EOp b;
        b.form = F_M4;
        b.q = e.q;
        b.c = e.q + n;
        b.mat = (int)mats.size();
        b.gate = e.gate;
        mats.push_back(superop(uu, 1));
        dm.push_back(b);
    }
    // plan and upload through the handle's own path with the superoperator circuit
    s->mats.swap(mats);
    return set_circuit_lowered(s, dm, gates, n_gates, 0.0);
}

svb_status svb_dm_probabilities(svb_sim* s, double* out)
{
    if (!s || !out) { set_error("svb_dm_probabilities: NULL argument"); return SVB_ERR_INVALID; }
    if (!s->dm_qubits) { set_error("svb_dm_probabilities: not a density-matrix handle"); return SVB_ERR_STATE; }
    const int n = (int)s->dm_qubits;
    const uint64_t dim = 1ull << n;
    cudaError_t e = cudaSetDevice(s->device);
    double* d = nullptr;
    if (e == cudaSuccess) e = cudaMalloc(&d, dim * sizeof(double));
    if (e == cudaSuccess) {
        const unsigned grid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((dim + 255) / 256, 148ull * 8));
        k_dm_diag<double><<<grid, 256>>>(static_cast<const double2*>(s->state), dim, n, d);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(out, d, dim * sizeof(double), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) {
        set_error(std::string("svb_dm_probabilities: ") + cudaGetErrorString(e));
        (void)cudaGetLastError();
        return SVB_ERR_CUDA;
    }
    return SVB_OK;
}

}  // extern "C"
