// cpd64.cpp -- command-line driver with the reference cpd64's flags and
// output lines (src/main.cpp:70-96, 322-390), running the GPU path through
// the C ABI of libblco_b200.
//
//   cpd64 -i X.tns -k 10 -r 16 -m 20 -e 1e-5 [-o out] [-x seed]
//   cpd64 -i X.tns -k 1 -p -t 0 -m 5          MTTKRP benchmark
//   cpd64 -i X.tns -k 1 -c -p -t 0            MTTKRP check against COO
//
// Differences from the reference, by design:
//   * every error is reported and the exit code is non-zero (the reference
//     exits inside check_cuda, src/utils.cu:131-137);
//   * -k 0 (the CPU ALTO path) and -d/-s (the Poisson generator) are not
//     provided: this engine is the GPU path only;
//   * --max_block_size is accepted as a spelling of --max-block-size.
#include <getopt.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <string>
#include <thread>
#include <vector>

#include "blco.h"
#include "tns_io.h"

using namespace blco_host;

static void usage(const char* call)
{
    fprintf(stderr, "Usage: %s [OPTIONS]\n", call);
    fprintf(stderr, "Options:\n");
    fprintf(stderr, "\t-h or --help         Display this information\n");
    fprintf(stderr, "\t-v or --version      Display version information\n");
    fprintf(stderr, "\t-i or --input        Input tensor file in text\n");
    fprintf(stderr, "\t-o or --output       Output tensor to file\n");
    fprintf(stderr, "\t-b or --bin          Input tensor file in binary\n");
    fprintf(stderr, "\t-f or --file         Save tensor to another format\n");
    fprintf(stderr, "\t-r or --rank         Rank\n");
    fprintf(stderr, "\t-m or --max-iter     Maximum outter iterations\n");
    fprintf(stderr, "\t-t or --target-mode  Target mode of tensor\n");
    fprintf(stderr, "\t-e or --epsilon      Convergence criteria\n");
    fprintf(stderr, "\t-x or --seed         Random value seed\n");
    fprintf(stderr, "\t-c or --check        Check GPU MTTKRP against sequential COO MTTKRP\n");
    fprintf(stderr, "\t-p or --bench        Run the GPU MTTKRP benchmark\n");
    fprintf(stderr, "\t-k or --kernel-id    ID of the GPU kernel to run (10 for auto)\n");
    fprintf(stderr, "\t-n or --num-partitions Number of partitions\n");
    fprintf(stderr, "\t--device             CUDA device ordinal\n");
    fprintf(stderr, "\t--thread-cf          Thread coarsening factor\n");
    fprintf(stderr, "\t--stream-data        Stream data to the GPU during computation\n");
    fprintf(stderr, "\t--max-block-size     Block size (nonzeros) on the GPU\n");
    fprintf(stderr, "\t--batch              Accepted for compatibility (blocks always run in one launch)\n");
    fprintf(stderr, "\t--selector FILE      Trained schedule selector (selector_params.bin) for -k 21\n");
    fprintf(stderr, "\t--host-load          Parse the .tns file on the host (default: on the GPU, except with -c / -f)\n");
    fprintf(stderr, "\t--precision P        CP-ALS numeric form: fp64 (default, the reference's), mixed (FP32\n"
                    "\t                     values and gathers, FP64 solve and fit) or mixed-bf16 (BF16 gathers)\n");
}

// Reads a selector parameter file (int32 hidden width, int32 count, then
// float32 parameters, little-endian) and makes it the network of kernel 21.
static bool load_selector(const std::string& path, int device, blco_mlp** out, std::string* err)
{
    FILE* f = fopen(path.c_str(), "rb");
    if (!f) { *err = "cannot open " + path; return false; }
    int32_t hdr[2] = {0, 0};
    bool ok = fread(hdr, sizeof(int32_t), 2, f) == 2 && hdr[0] > 0 && hdr[1] > 0;
    std::vector<float> params(ok ? (size_t)hdr[1] : 0);
    ok = ok && fread(params.data(), sizeof(float), params.size(), f) == params.size();
    fclose(f);
    if (!ok) { *err = "malformed selector file " + path; return false; }
    blco_mlp* net = nullptr;
    int n = 0;
    if (blco_mlp_create(hdr[0], 0, device, &net) != BLCO_OK || blco_mlp_num_params(net, &n) != BLCO_OK ||
        n != hdr[1] || blco_mlp_set_params(net, params.data(), n) != BLCO_OK) {
        *err = std::string("selector: ") + blco_last_error();
        if (net) blco_mlp_destroy(net);
        return false;
    }
    blco_selector_set(net, 0.1f);
    *out = net;
    return true;
}

static void print_tensor_info(uint64_t rank, int max_iters, const Coo& X, uint64_t nnz)
{
    // PrintTensorInfo (src/main.cpp:756-778)
    double cells = 1.0;
    for (auto d : X.dims) cells *= (double)d;
    fprintf(stderr, "# Modes         = %u\n", (unsigned)X.nmodes);
    fprintf(stderr, "Rank            = %llu\n", (unsigned long long)rank);
    fprintf(stderr, "Sparsity        = %f\n", (double)nnz / cells);
    fprintf(stderr, "Max iters       = %d\n", max_iters);
    fprintf(stderr, "Dimensions      = [%llu", (unsigned long long)X.dims[0]);
    for (int i = 1; i < X.nmodes; i++) fprintf(stderr, " X %llu", (unsigned long long)X.dims[i]);
    fprintf(stderr, "]\n");
    fprintf(stderr, "NNZ             = %llu\n", (unsigned long long)nnz);
}

// Sequential COO MTTKRP, the reference's -c ground truth
// (include/cpd.hpp:510-544): U[mode] += MTTKRP.
static void coo_mttkrp(const Coo& X, Kruskal& M, int mode)
{
    const int R = M.rank;
    std::vector<double> row(R);
    for (uint64_t i = 0; i < X.nnz(); i++) {
        for (int r = 0; r < R; r++) row[r] = X.vals[i];
        for (int m = 0; m < X.nmodes; m++) {
            if (m == mode) continue;
            const double* u = &M.U[m][X.cidx[m][i] * R];
            for (int r = 0; r < R; r++) row[r] *= u[r];
        }
        double* o = &M.U[mode][X.cidx[mode][i] * R];
        for (int r = 0; r < R; r++) o[r] += row[r];
    }
}

// VerifyResult (src/main.cpp:652-675)
static bool verify(const char* name, const std::vector<double>& truth, const std::vector<double>& got)
{
    uint64_t cnt = 0;
    for (size_t i = 0; i < truth.size(); i++) {
        double moe = std::max(std::fabs(truth[i]) * 1e-6, 1e-6);
        if (std::fabs(truth[i] - got[i]) > moe) cnt++;
    }
    if (cnt == 0) fprintf(stderr, "Results of %s is correct\n", name);
    else fprintf(stderr, "Results of %s is incorrect by %llu\n", name, (unsigned long long)cnt);
    return cnt == 0;
}

static int die(const char* what, int st)
{
    fprintf(stderr, "Error: %s: %s (%s)\n", what, blco_last_error(), blco_status_string(st));
    return 2;
}

int main(int argc, char** argv)
{
    static const struct option long_opt[] = {
        {"help", 0, nullptr, 'h'},       {"version", 0, nullptr, 'v'},     {"input", 1, nullptr, 'i'},
        {"output", 1, nullptr, 'o'},     {"bin", 1, nullptr, 'b'},         {"rank", 1, nullptr, 'r'},
        {"max-iter", 1, nullptr, 'm'},   {"seed", 1, nullptr, 'x'},        {"dims", 1, nullptr, 'd'},
        {"target-mode", 1, nullptr, 't'}, {"sparsity", 1, nullptr, 's'},   {"epsilon", 1, nullptr, 'e'},
        {"file", 1, nullptr, 'f'},       {"check", 0, nullptr, 'c'},       {"bench", 0, nullptr, 'p'},
        {"kernel-id", 1, nullptr, 'k'},  {"num-partitions", 1, nullptr, 'n'}, {"device", 1, nullptr, 1001},
        {"thread-cf", 1, nullptr, 1002}, {"stream-data", 0, nullptr, 1003}, {"max-block-size", 1, nullptr, 1004},
        {"max_block_size", 1, nullptr, 1004}, {"batch", 0, nullptr, 1005}, {"selector", 1, nullptr, 1006},
        {"host-load", 0, nullptr, 1007}, {"precision", 1, nullptr, 1008},
        {nullptr, 0, nullptr, 0}};
    int max_iters = 10;
    long long rank = 16;
    int target_mode = 0;
    std::string text_file, out_file, bin_file, selector_file;
    double epsilon = 1e-5;
    int seed = (int)time(nullptr);
    int save_to_file = 0;
    bool do_check = false, do_bench = false, stream_data = false, want_dims = false, host_load = false;
    int kernel_id = 0;
    const char* omp = getenv("OMP_NUM_THREADS");
    int nthreads = omp && atoi(omp) > 0 ? atoi(omp) : (int)std::max(1u, std::thread::hardware_concurrency());
    int num_partitions = nthreads;
    int device = 0, thread_cf = 2;
    int precision = BLCO_PRECISION_FP64;
    long long max_block_size = 16777216;
    int c;
    while ((c = getopt_long(argc, argv, "hvi:o:b:r:m:x:d:t:s:e:f:cpk:n:", long_opt, nullptr)) != -1) {
        switch (c) {
        case 'h': usage(argv[0]); return 0;
        case 'v': printf("%s version %s\n", argv[0], blco_version()); return 0;
        case 'i': text_file = optarg; break;
        case 'o': out_file = optarg; break;
        case 'b': bin_file = optarg; break;
        case 'r': rank = atoll(optarg); if (rank < 1) { fprintf(stderr, "Invalid -rank: %s.\n", optarg); return 1; } break;
        case 'm': max_iters = atoi(optarg); if (max_iters < 0) { fprintf(stderr, "Invalid -max-iter: %s.\n", optarg); return 1; } break;
        case 'x': seed = atoi(optarg); if (seed < 0) { fprintf(stderr, "Invalid -seed: %s.\n", optarg); return 1; } break;
        case 'd': want_dims = true; break;
        case 't': target_mode = atoi(optarg); if (target_mode < -1) { fprintf(stderr, "Invalid -target-mode: %s.\n", optarg); return 1; } break;
        case 's': break;
        case 'e': epsilon = atof(optarg); if (epsilon < 0) { fprintf(stderr, "Invalid -epsilon: %s.\n", optarg); return 1; } break;
        case 'f': save_to_file = atoi(optarg); break;
        case 'c': do_check = true; break;
        case 'p': do_bench = true; break;
        case 'k': kernel_id = atoi(optarg); if (kernel_id < 0) { fprintf(stderr, "Invalid -kernel-id: %s.\n", optarg); return 1; } break;
        case 'n': num_partitions = atoi(optarg); if (num_partitions <= 0) { fprintf(stderr, "Invalid -num-partitions: %s.\n", optarg); return 1; } break;
        case 1001: device = atoi(optarg); if (device < 0) { fprintf(stderr, "Invalid -device: %s.\n", optarg); return 1; } break;
        case 1002: thread_cf = atoi(optarg); if (thread_cf <= 0) { fprintf(stderr, "Invalid -thread-cf: %s.\n", optarg); return 1; } break;
        case 1003: stream_data = true; break;
        case 1004: max_block_size = atoll(optarg); if (max_block_size <= 0) { fprintf(stderr, "Invalid -max-block-size: %s.\n", optarg); return 1; } break;
        case 1005: break;
        case 1006: selector_file = optarg; break;
        case 1007: host_load = true; break;
        case 1008:
            if (!strcmp(optarg, "fp64")) precision = BLCO_PRECISION_FP64;
            else if (!strcmp(optarg, "mixed")) precision = BLCO_PRECISION_MIXED;
            else if (!strcmp(optarg, "mixed-bf16")) precision = BLCO_PRECISION_MIXED_BF16;
            else { fprintf(stderr, "Invalid -precision: %s (fp64, mixed or mixed-bf16).\n", optarg); return 1; }
            break;
        default: usage(argv[0]); return 1;
        }
    }
    if (precision != BLCO_PRECISION_FP64 && (do_check || do_bench)) {
        fprintf(stderr, "--precision selects the CP-ALS form; the -c / -p MTTKRP runs are FP64.\n");
        return 1;
    }
    Coo X;
    std::string err;
    if (kernel_id != 0 && do_check) max_iters = 1;
    if (!stream_data) max_block_size = 0; // one block (src/main.cpp:327)
    blco_opts opts;
    blco_opts_init(&opts);
    opts.kernel = kernel_id;
    opts.nprtn = num_partitions;
    opts.thread_cf = thread_cf;
    opts.stream_data = stream_data ? 1 : 0;
    opts.precision = precision;
    opts.verbose = 1;
    opts.device = device;
    // The text file is parsed and encoded on the GPU unless the host COO
    // arrays are needed (-c check, -f conversion) or --host-load is given.
    const bool gpu_load = !text_file.empty() && bin_file.empty() && !do_check && !save_to_file && !host_load &&
                          kernel_id != 0;
    blco_tensor* T = nullptr;
    uint64_t nnz = 0;
    auto t0 = std::chrono::steady_clock::now();
    if (gpu_load) {
        blco_tns_info ti;
        int st = blco_encode_tns(text_file.c_str(), (uint64_t)max_block_size, &opts, &T, &ti);
        if (st) {
            fprintf(stderr, "Error: %s\n", blco_last_error());
            return 1;
        }
        X.nmodes = ti.nmodes;
        X.dims.assign(ti.dims, ti.dims + ti.nmodes);
        nnz = ti.nnz;
    } else if (!bin_file.empty()) {
        if (!read_bin(bin_file, &X, &err)) { fprintf(stderr, "Error: %s\n", err.c_str()); return 1; }
        if (save_to_file && !write_tns(bin_file + ".tns", X, &err)) { fprintf(stderr, "Error: %s\n", err.c_str()); return 1; }
    } else if (!text_file.empty()) {
        if (!read_tns(text_file, &X, &err)) { fprintf(stderr, "Error: %s\n", err.c_str()); return 1; }
        if (save_to_file && !write_bin(text_file + ".bin", X, &err)) { fprintf(stderr, "Error: %s\n", err.c_str()); return 1; }
    } else {
        if (want_dims) fprintf(stderr, "The synthetic Poisson generator (-d/-s) is not part of this engine.\n");
        else fprintf(stderr, "No dims specified... exiting\n");
        usage(argv[0]);
        return 1;
    }
    if (!gpu_load) nnz = X.nnz();
    double t_read = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    printf("[%s]: %.6f s\n", "Reading tensor file", t_read);
    if (kernel_id == 0) {
        fprintf(stderr, "The CPU ALTO path is not part of this engine: pass -k (10 = automatic kernel).\n");
        return 1;
    }
    if (target_mode >= X.nmodes || target_mode < 0) {
        fprintf(stderr, "Invalid -target-mode: %d.\n", target_mode);
        if (T) blco_tensor_free(T);
        return 1;
    }

    blco_mlp* selector = nullptr;
    if (!selector_file.empty() && !load_selector(selector_file, device, &selector, &err)) {
        fprintf(stderr, "Error: %s\n", err.c_str());
        return 1;
    }
    if (gpu_load) {
        printf("BLCO: encode time = %f (s) (parsed and encoded on the GPU with the file)\n", t_read);
    } else {
        std::vector<const uint64_t*> cptr(X.nmodes);
        for (int n = 0; n < X.nmodes; n++) cptr[n] = X.cidx[n].data();
        auto te = std::chrono::steady_clock::now();
        int st = blco_encode(X.nmodes, X.dims.data(), X.nnz(), cptr.data(), X.vals.data(), (uint64_t)max_block_size,
                             &opts, &T);
        if (st) return die("BLCO encode", st);
        printf("BLCO: encode time = %f (s)\n", std::chrono::duration<double>(std::chrono::steady_clock::now() - te).count());
    }
    blco_tensor_info info;
    blco_tensor_get_info(T, &info);
    printf("Total blocks: %llu\n\n", (unsigned long long)info.block_count);
    int st = BLCO_OK;

    print_tensor_info((uint64_t)rank, max_iters, X, nnz);
    Kruskal M;
    M.nmodes = X.nmodes;
    M.rank = (int)rank;
    M.dims = X.dims;
    kruskal_random_init(&M, (unsigned)seed, nthreads);
    std::vector<double*> uptr(X.nmodes);
    for (int n = 0; n < X.nmodes; n++) uptr[n] = M.U[n].data();

    int rc = 0;
    if (do_bench || do_check) {
        // mttkrp_alto_dev (src/alto_dev.cu:1857-1952): the output is the
        // target factor itself and accumulates over the iterations.
        std::vector<std::vector<double>> truth;
        if (do_check) {
            Kruskal Mt = M;
            printf("===Do base run===\n");
            coo_mttkrp(X, Mt, target_mode);
            printf("--> MTTKRP sequential base run done.\n");
            truth = Mt.U;
            printf("===Do GPU run===\n");
        }
        double total_ms = 0.0;
        for (int it = 0; it < max_iters; it++) {
            auto a = std::chrono::steady_clock::now();
            st = blco_mttkrp_host(T, target_mode, (int)rank, uptr.data(), uptr[target_mode], &opts);
            if (st) return die("MTTKRP", st);
            total_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - a).count();
        }
        printf("Total time for MTTKRP: %0.3f (time per iter: %0.3f ms)\n", total_ms,
               max_iters ? total_ms / max_iters : 0.0);
        if (do_check) {
            printf("MTTKRP GPU run done.\n");
            printf("===Verify GPU MTTKRP=== (target mode: %d)\n", target_mode);
            for (int m = 0; m < X.nmodes; m++) {
                printf("mode %d: ", m);
                fflush(stdout);
                if (!verify("mttkrp_blco_dev", truth[m], M.U[m])) rc = 3;
            }
        }
    } else {
        double fit = 0.0;
        int iters = 0;
        printf("\nCopying to GPU device\n");
        st = blco_cpals(T, (int)rank, uptr.data(), M.lambda.data(), max_iters, epsilon, &opts, &fit, nullptr, &iters);
        if (st) return die("CP-ALS", st);
        if (!out_file.empty()) {
            if (!export_kruskal(M, out_file, &err)) { fprintf(stderr, "Error: %s\n", err.c_str()); return 1; }
            printf("--> Kruskal model saved to %s\n", out_file.c_str());
        }
    }
    blco_tensor_free(T);
    if (selector) {
        blco_selector_set(nullptr, 0.f);
        blco_mlp_destroy(selector);
    }
    return rc;
}
