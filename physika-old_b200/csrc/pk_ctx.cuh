// pk_ctx.cuh -- the context object behind the opaque pk_ctx handle.
#pragma once
#include <string>
#include <vector>

#include "pk_internal.cuh"

struct pk_ctx {
    int device = 0;
    std::string err;
    int* d_err = nullptr;  // latched device-side conditions (kErr* bits)
    int launches = 0;      // kernels enqueued by the last fused step

    // ---- optional per-kernel-class event timing (pk_ctx_profile)
    bool prof = false;
    std::vector<cudaEvent_t> prof_ev[PK_PROF_KINDS];  // start/stop pairs
    int prof_used[PK_PROF_KINDS] = {0, 0, 0, 0, 0, 0};

    // ---- particle-sized scratch (capacity cap_n)
    int cap_n = 0;
    int* perm = nullptr;
    int* inv = nullptr;
    int* key = nullptr;
    int* rank = nullptr;
    int* count = nullptr;     // hits per particle (sorted order)
    int* count_c = nullptr;   // hits per particle (caller order, dynamic lists)
    int* offs = nullptr;      // exclusive scan of count_c (n + 1)
    int* hcnt = nullptr;      // hits per particle in the hit rows (sorted order)
    int2* items = nullptr;    // list-build work items: sorted ranges sharing one cell
    int* nitems = nullptr;    // device counter of items (1 int)
    float4* xs_pre = nullptr;
    float4* xs0 = nullptr;
    float4* xa = nullptr;
    float4* xb = nullptr;     // (x, lambda) written by pass A
    float4* vs = nullptr;
    float4* vv = nullptr;     // sorted velocities of the viscosity sweeps
    float* rho = nullptr;
    int2* rcnt = nullptr;
    uint2* tau = nullptr;
    unsigned* tau_hint = nullptr;  // caller order: d2 bits of the last frame's tau (selection pivot)

    // ---- rows (capacity cap_rows entries: row_cap per particle)
    long long cap_rows = 0;
    int* rows = nullptr;      // solver rows: sorted index | flag bits
    uint2* hits = nullptr;    // hit rows: (sorted index, d2 bits), candidate order
    // Entries of a particle past row_cap (hits and solver row alike) go to the
    // spill pool: ovf[s] is the particle's segment, holding round4(count -
    // row_cap) entries of each array.  spill[0] counts the entries handed out
    // in the last build (also past pool_cap: the size the next build grows the
    // pool to), spill[1] the particles listed in ovf_list.
    long long pool_cap = 0;
    long long pool_need = 0;  // entries the last synchronised build asked for
    uint2* hpool = nullptr;
    int* rpool = nullptr;
    int* tile_cnt = nullptr;  // persistent passes: tiles per scene (n + 2)
    int* tile_off = nullptr;  // their exclusive scan (n + 2; [nscenes + 1] = tiles)
    int2* tiles = nullptr;    // sorted ranges of the tiles (n + n/128 + 2)
    int* ovf = nullptr;       // per sorted particle (valid where its count > row_cap)
    int* ovf_list = nullptr;  // sorted particles with a spill segment
    unsigned long long* spill = nullptr;  // 2 device counters

    // ---- dense cell table (capacity cap_keys entries + 2)
    long long cap_keys = 0;
    int* cell_cnt = nullptr;
    int* cell_start = nullptr;
    int* scan_part = nullptr;  // block partials of the scan
    long long cap_part = 0;

    // ---- generic-list solver scratch (caller order)
    int cap_g = 0;
    float* g_rho = nullptr;
    float* g_lam = nullptr;
    float* g_dpos = nullptr;  // 3 per particle
    float* g_xold = nullptr;  // 3 per particle
    // device copies of the caller's host arrays (pk_pbf_step_host)
    float* h_x = nullptr;  // 3 per particle
    float* h_v = nullptr;  // 3 per particle
    int h_cap = 0;

    // ---- a recorded frame (pk_graph_capture)
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    cudaStream_t capture_stream = nullptr;

    // ---- state of the last neighbour build
    pk::Grid grid{};
    int nq_n = -1;
    int nq_cap = 0;
    int row_cap = 0;
    float nq_h = 0.0f;
    const int* exported_index = nullptr;
    const int* exported_elements = nullptr;
    bool nq_valid = false;

    // ---- box boundary (BoundaryConstraint)
    float* sdf = nullptr;
    size_t sdf_bytes = 0;
    float sdf_left[3] = {0, 0, 0};
    float sdf_h[3] = {0, 0, 0};
    float sdf_box_lo[3] = {0, 0, 0};
    float sdf_box_hi[3] = {0, 0, 0};
    int sdf_dims[3] = {0, 0, 0};
    int sdf_inverted = 1;
    bool has_sdf = false;

    // ---- peridynamics (ElasticityModule) frozen state
    int pd_n = -1;
    int pd_cap = 0;            // layout of the rest shape (0 = CSR)
    long long pd_total = 0;
    int* pd_index = nullptr;   // copy of the list index (counts or offsets)
    int* pd_rest_idx = nullptr;
    float* pd_rest_pos = nullptr;  // 3 per bond
    unsigned char* pd_alive = nullptr;
    float* pd_invK = nullptr;      // 9 per particle, row-major
    float* pd_bulk = nullptr;
    float* pd_xold = nullptr;
    float* pd_delta = nullptr;
    float* pd_w = nullptr;
    float* pd_ktw = nullptr;  // computeInverseK: the weight sum between its two kernels
    float pd_horizon = 0.0f;
    long long pd_cap_bonds = 0;    // capacity of pd_alive and pd_in
    long long pd_cap_rest = 0;     // capacity of pd_rest_idx / pd_rest_pos
    int pd_cap_n = 0;
    // ElastoplasticityModule state (n per array) and the spare rest-shape
    // buffers a reconstruction fills before they are swapped in
    int pl_cap_n = 0;
    float* pl_y1 = nullptr;         // m_yiled_I1
    float* pl_y2 = nullptr;         // m_yield_J2
    float* pl_i1 = nullptr;         // m_I1
    unsigned char* pl_yield = nullptr;  // m_bYield
    float* pl_invF = nullptr;       // m_invF, 9 per particle
    float* pl_mk = nullptr;         // rotateRestShape: sums, then the rotation (kPlMk per particle)
    int* pl_sizes = nullptr;        // n + 1
    int* pl_off = nullptr;          // n + 1
    int* pl_rest_idx2 = nullptr;
    float* pl_rest_pos2 = nullptr;
    long long pl_cap_rest2 = 0;
    bool pd_begun = false;          // pk_pd_begin has run since pk_pd_init
    // Autotuner of the frame kernels (pk_ctx_autotune): a few trial frames
    // time the pass block sizes and the build's particles per pass; the
    // choices change no result.
    struct Tune {
        bool on = false;
        int frame = 0;
        int pass_block = 256;   // Jacobi pass threads per block: 128, 256, 512
        bool persist = false;   // Jacobi passes as a resident grid walking scene tiles
        int build_pb = 8;       // k_build particles per pass: 4, 8 or 16 (8 measured fastest at 2M)
        float pass_ms[4] = {0, 0, 0, 0};  // 128, 256, 512, 256 resident
        float build_ms[3] = {0, 0, 0};
        cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};  // build start/end, solve start/end
    } tune;
    int* pd_in_cnt = nullptr;   // incoming bonds per particle (n + 1)
    int* pd_in_off = nullptr;   // their CSR offsets (n + 1)
    int2* pd_in = nullptr;      // (source particle, bond slot) of every incoming bond
    int* pd_in_slot = nullptr;  // the bond slots alone, in the same order (the gathers' 4-byte stream)
    // projection workspaces (float, double) and the parameters of the last rollout
    void* pbd_roll = nullptr;   // differentiable DensityPBD rollout (pk_pbd_adj.cu)
    void* pd_work32 = nullptr;
    void* pd_work64 = nullptr;
    float pd_horizon_last = 0.f, pd_mu_last = 0.f, pd_lambda_last = 0.f;
};
