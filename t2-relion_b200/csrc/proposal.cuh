// Learned orientation proposals: shared constants and state (internal).
#pragma once
#include "t2b_internal.cuh"

namespace t2b {

constexpr int NET_NPIX = 256;      // 16 x 16 feature image
constexpr int NET_C1 = 16, NET_C2 = 32;
constexpr int NET_H0 = 2048, NET_H1 = 1024, NET_H2 = 1024;
constexpr int NET_RING = 8;        // Fourier rings read by the network
constexpr int NET_MAX_RING = 512;  // ring pixels of the window (|k| <= 8: 145)
constexpr int NET_NPOST = 8;       // posterior labels kept per training particle
constexpr int NET_NTGT = 1 + NET_NPOST;
constexpr int NET_TOPK_CAND = 2048;
constexpr int NET_MAX_KO = 49152;  // logits of one particle held in shared memory by the top-k
constexpr int NET_KSPLIT = 16;     // K slices of the fc1 / fc2 inference GEMMs
constexpr int NET_MAX_K1 = 1024;   // network candidates rescored at low resolution

// offsets (elements) of the parameters in the flat FP32 / BF16 vectors;
// w3 last, with zero rows up to a multiple of 128 for the tensor-core operand
struct NetLayout {
    size_t wc1, bc1, wc2, bc2, b1, b2, b3, w1, w2, w3, total, alloc;
    int KO, KOpad;
};
NetLayout net_layout(int KO);

struct PropState {        // device
    int gate;             // 1: the batch's coarse pass runs on the proposals
    int na;               // audited particles of the batch
    long long seen;       // particles of the stream so far
};

struct GenParams {
    unsigned long long seed;
    double dmin, dmax, astig, kv, cs, q0, angpix, max_shift;
    const float* minv;    // device, P: noise model (1/sigma^2 per pixel, 0 = no noise)
};

struct ProposalNet {
    NetLayout L{};
    int KO = 0;
    bool trained = false;
    long long adam_t = 0;
    std::vector<void*> owned;          // parameters and optimiser state
    std::vector<void*> ws;             // per-configuration workspace below
    float *th = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;
    void* thb = nullptr;               // BF16 copy of th (every forward pass reads it)
    bool ready = false;                // workspace matches the configuration
    bool enabled = false;
    int kprop = 64, every = 50, na_max = 0, kslot = 128, tn = 96, b_pad = 0;
    int k1 = 0;                        // network candidates rescored at low resolution (0: none)
    int kr = 0;                        // K of the rescoring contraction (2 x ring pixels, padded)
    float2* projR = nullptr;           // K*O x nring: projections at the ring pixels (FP32)
    void *rth = nullptr, *rtl = nullptr;  // K*O x kr: the same, split-BF16
    float* w2r = nullptr;              // B x nring
    void *rah = nullptr, *ral = nullptr;  // B*NET_MAX_K1 x kr: gathered candidate rows
    void *rbh = nullptr, *rbl = nullptr;  // B*T x kr: shifted ring images
    float* rnorm = nullptr;            // B*K1 ring norms
    int* cand1 = nullptr;              // B x k1 network candidates
    float* score1 = nullptr;           // B x k1 low-resolution scores
    double thr = 0.999;
    int nring = 0;
    int *ring = nullptr, *ring_k = nullptr;
    float* img = nullptr;
    void *x0b = nullptr, *h1b = nullptr, *h2b = nullptr;
    float *y1 = nullptr, *y2 = nullptr, *logits = nullptr;
    int* prop = nullptr;
    void* maps = nullptr;              // 6 tensor maps: W1, X0b, W2, H1b, W3, H2b
    void *pg_h = nullptr, *pg_l = nullptr;
    void *ab_h = nullptr, *ab_l = nullptr;   // phase rows ab_t of the translations (split-BF16, tn rows)
    float* part = nullptr;                   // split-K partial accumulators of the proposal tiles
    int* fix = nullptr;                      // and their arrival counters
    int part_tiles = 0;                      // m-tiles they cover
    int pg_rows = 0;                         // rows of the proposal A operand (K-blocked)
    float* nprop = nullptr;
    PropState* ps = nullptr;
    int* audit_b = nullptr;
    void *ia_h = nullptr, *ia_l = nullptr;
    float *c0a = nullptr, *norma = nullptr, *d2a = nullptr;
    void *wa_h = nullptr, *wa_l = nullptr;   // w2 of the audit slots (split-BF16, kn wide, 32-row padded)
    unsigned* minkeya = nullptr;
    double* asum = nullptr;
};

// inference, audit and restricted coarse pass of one batch (proposal.cu)
void proposal_infer(t2b_ctx* c, const Work& w, cudaStream_t st);
// ev (optional): two events recorded around the audit / proposal contraction.
// proposal_audit = proposal_audit_contract (audited particles, their operands, norms and full
// contraction: needs the prepared images only) then proposal_audit_mass (the posterior mass
// inside the proposals, the gate: needs proposal_infer's proposals).
void proposal_audit(t2b_ctx* c, const Work& w, cudaStream_t st, cudaEvent_t* ev = nullptr);
void proposal_audit_contract(t2b_ctx* c, const Work& w, cudaStream_t st, cudaEvent_t* ev = nullptr);
void proposal_audit_mass(t2b_ctx* c, const Work& w, cudaStream_t st);
void proposal_coarse(t2b_ctx* c, const Work& w, cudaStream_t st, cudaEvent_t* ev = nullptr);
void proposal_release(t2b_ctx* c);    // context destruction
void proposal_invalidate(t2b_ctx* c); // configuration changed

}  // namespace t2b
