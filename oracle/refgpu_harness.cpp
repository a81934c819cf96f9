// TEST INFRASTRUCTURE ONLY: drives QUICK's own CUDA get2e through its C entry
// points, exactly in the order QUICK's Fortran makes the calls, and times it.
//
// Call order (src/gpu/cuda/gpu.h:14-111; scf_operator,
// src/modules/quick_scf_operator_module.f90:94-153):
//   gpu_new_ -> gpu_init_device_ -> gpu_setup_ -> gpu_upload_method_ ->
//   gpu_upload_xyz_ -> gpu_upload_atom_and_chg_ -> gpu_upload_basis_ ->
//   gpu_upload_cutoff_matrix_ -> gpu_allocate_scratch_, then per Fock build
//   gpu_upload_calculated_ -> gpu_upload_cutoff_ -> gpu_get_cshell_eri_.
//
// Usage: refgpu_get2e <input.bin> <G_out.bin> <steps> <warmup>
// The input file is written by oracle/refgpu.py (layout documented there).  The
// program prints one JSON line: per-build times of the whole per-iteration call
// sequence (host wall clock; the reference's calls are synchronous) and of the
// get2e kernels alone (CUDA events), and whether two builds gave the same bits.
// gpu_delete_ resets the device, so this always runs as its own process.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include <cuda_runtime.h>

extern "C" {
void gpu_new_(int*);
void gpu_init_device_(int*);
void gpu_setup_(int*, int*, int*, int*, int*, int*);
void gpu_upload_method_(int*, bool*, double*);
void gpu_upload_xyz_(double*);
void gpu_upload_atom_and_chg_(int*, double*);
void gpu_upload_basis_(int*, int*, int*, int*, int*, int*, int*, double*, double*, int*, int*, int*, int*, int*,
                       int*, int*, int*, int*, int*, int*, int*, int*, int*, int*, int*, double*, double*, double*,
                       int*);
void gpu_upload_cutoff_matrix_(double*, double*);
void gpu_allocate_scratch_(bool*);
void gpu_deallocate_scratch_(bool*);
void gpu_upload_calculated_(double*, double*, double*, double*);
void gpu_upload_cutoff_(double*, double*, double*, double*, double*);
void gpu_get_cshell_eri_(bool*, double*);
void gpu_delete_(int*);
int refgpu_time_get2e(int nrep, void* flush, size_t flush_bytes, float* ms);
}

namespace {

struct Reader {
    FILE* f;
    template <typename T>
    std::vector<T> get(size_t n) {
        std::vector<T> v(n);
        if (n && std::fread(v.data(), sizeof(T), n, f) != n) {
            std::fprintf(stderr, "refgpu harness: input file too short\n");
            std::exit(2);
        }
        return v;
    }
};

double median(std::vector<double> v) {
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    return v[v.size() / 2];
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 5) {
        std::fprintf(stderr, "usage: %s input.bin G_out.bin steps warmup\n", argv[0]);
        return 2;
    }
    const int steps = std::atoi(argv[3]), warmup = std::atoi(argv[4]);
    FILE* f = std::fopen(argv[1], "rb");
    if (!f) { std::perror(argv[1]); return 2; }
    Reader R{f};
    // header: 12 int32 then 2 float64
    auto hdr = R.get<int>(12);
    int natom = hdr[0], nbasis = hdr[1], nshell = hdr[2], nprim = hdr[3], jbasis = hdr[4], maxcontract = hdr[5];
    const int maxprim = hdr[6];
    int nelec = hdr[7], imult = 1, molchg = hdr[8], iattype_first = 1;
    auto cuts = R.get<double>(2);
    double integralCutoff = cuts[0], primLimit = cuts[1];
    double dmCutoff = 1e-10, coreCutoff = 1e-12;
    auto xyz = R.get<double>(3 * (size_t)natom);
    auto chg = R.get<double>(natom);
    auto iattype = R.get<int>(natom);
    auto ncontract = R.get<int>(nbasis);
    auto itype = R.get<int>(3 * (size_t)nbasis);
    auto aexp = R.get<double>((size_t)maxcontract * nbasis);
    auto dcoeff = R.get<double>((size_t)maxcontract * nbasis);
    auto ncenter = R.get<int>(nbasis);
    auto kstart = R.get<int>(nshell);
    auto katom = R.get<int>(nshell);
    auto ktype = R.get<int>(nshell);
    auto kprim = R.get<int>(nshell);
    auto ksumtype = R.get<int>(nshell + 1);
    auto qnumber = R.get<int>(nshell);
    auto qstart = R.get<int>(nshell);
    auto qfinal = R.get<int>(nshell);
    auto qsbasis = R.get<int>(4 * (size_t)nshell);
    auto qfbasis = R.get<int>(4 * (size_t)nshell);
    auto gccoeff = R.get<double>((size_t)maxprim * nbasis);
    auto cons = R.get<double>(nbasis);
    auto gcexpo = R.get<double>((size_t)maxprim * nbasis);
    auto klmn = R.get<int>(3 * (size_t)nbasis);
    auto Y = R.get<double>((size_t)nshell * nshell);
    auto cutprim = R.get<double>((size_t)jbasis * jbasis);
    auto D = R.get<double>((size_t)nbasis * nbasis);
    auto cutmat = R.get<double>((size_t)nshell * nshell);
    std::fclose(f);
    (void)iattype_first;

    int ierr = 0;
    gpu_new_(&ierr);
    gpu_init_device_(&ierr);
    if (ierr) { std::fprintf(stderr, "refgpu harness: gpu_init_device_ ierr %d\n", ierr); return 3; }
    int iAtomType = 1;
    gpu_setup_(&natom, &nbasis, &nelec, &imult, &molchg, &iAtomType);
    int method = 0;
    bool oshell = false;
    double hyb = 1.0;
    gpu_upload_method_(&method, &oshell, &hyb);
    gpu_upload_xyz_(xyz.data());
    gpu_upload_atom_and_chg_(iattype.data(), chg.data());
    // unused by the reference (its uploads of these are commented out): placeholders
    std::vector<int> unused_atom(std::max(natom, 1), 0), unused_shell(std::max(nshell, 1), 0), kshell(93, 0);
    int jshell = nshell;
    int maxc = maxcontract;
    auto t_setup0 = std::chrono::steady_clock::now();
    gpu_upload_basis_(&nshell, &nprim, &jshell, &jbasis, &maxc, ncontract.data(), itype.data(), aexp.data(),
                      dcoeff.data(), unused_atom.data(), unused_atom.data(), unused_shell.data(),
                      unused_shell.data(), ncenter.data(), kstart.data(), katom.data(), ktype.data(), kprim.data(),
                      kshell.data(), ksumtype.data(), qnumber.data(), qstart.data(), qfinal.data(), qsbasis.data(),
                      qfbasis.data(), gccoeff.data(), cons.data(), gcexpo.data(), klmn.data());
    gpu_upload_cutoff_matrix_(Y.data(), cutprim.data());
    bool grad_scratch = false;
    gpu_allocate_scratch_(&grad_scratch);
    cudaDeviceSynchronize();
    const double setup_s =
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t_setup0).count();

    const size_t nn = (size_t)nbasis * nbasis;
    std::vector<double> o(nn, 0.0), G1(nn, 0.0), G2(nn, 0.0);
    bool deltaO = false;
    auto one_build = [&](std::vector<double>& out) {
        std::fill(out.begin(), out.end(), 0.0);
        gpu_upload_calculated_(out.data(), out.data(), out.data(), D.data());
        gpu_upload_cutoff_(cutmat.data(), &integralCutoff, &primLimit, &dmCutoff, &coreCutoff);
        gpu_get_cshell_eri_(&deltaO, out.data());
    };
    one_build(G1);

    // the whole per-iteration call sequence, as QUICK's SCF makes it
    for (int w = 0; w < warmup; ++w) one_build(o);
    std::vector<double> seq_ms;
    for (int s = 0; s < steps; ++s) {
        std::fill(o.begin(), o.end(), 0.0);
        auto t0 = std::chrono::steady_clock::now();
        gpu_upload_calculated_(o.data(), o.data(), o.data(), D.data());
        gpu_upload_cutoff_(cutmat.data(), &integralCutoff, &primLimit, &dmCutoff, &coreCutoff);
        gpu_get_cshell_eri_(&deltaO, o.data());
        seq_ms.push_back(1e3 * std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count());
    }

    // the get2e kernels alone (CUDA events, L2 flushed before every build)
    void* flush = nullptr;
    const size_t flush_bytes = 256ull << 20;
    cudaMalloc(&flush, flush_bytes);
    gpu_upload_calculated_(G2.data(), G2.data(), G2.data(), D.data());
    gpu_upload_cutoff_(cutmat.data(), &integralCutoff, &primLimit, &dmCutoff, &coreCutoff);
    std::vector<float> kms(std::max(steps + warmup, 1), 0.f);
    const int rc = refgpu_time_get2e(steps + warmup, flush, flush_bytes, kms.data());
    std::fill(G2.begin(), G2.end(), 0.0);
    gpu_get_cshell_eri_(&deltaO, G2.data());
    cudaFree(flush);
    std::vector<double> kern(kms.begin() + warmup, kms.end());
    const bool same = std::memcmp(G1.data(), G2.data(), nn * sizeof(double)) == 0;
    const cudaError_t last = cudaGetLastError();

    FILE* g = std::fopen(argv[2], "wb");
    if (!g || std::fwrite(G1.data(), sizeof(double), nn, g) != nn) { std::perror(argv[2]); return 2; }
    std::fclose(g);
    double kmean = 0.0;
    for (double x : kern) kmean += x;
    kmean /= std::max<size_t>(1, kern.size());
    double smean = 0.0;
    for (double x : seq_ms) smean += x;
    smean /= std::max<size_t>(1, seq_ms.size());
    std::printf("{\"nbasis\": %d, \"setup_s\": %.6f, \"call_ms_mean\": %.6f, \"call_ms_median\": %.6f, "
                "\"kernel_ms_mean\": %.6f, \"kernel_ms_median\": %.6f, \"steps\": %d, \"warmup\": %d, "
                "\"bit_identical_repeat\": %s, \"timing_rc\": %d, \"cuda\": \"%s\"}\n",
                nbasis, setup_s, smean, median(seq_ms), kmean, median(kern), steps, warmup, same ? "true" : "false",
                rc, cudaGetErrorString(last));
    std::fflush(stdout);
    gpu_deallocate_scratch_(&grad_scratch);
    gpu_delete_(&ierr);
    return (rc == 0 && last == cudaSuccess) ? 0 : 4;
}
