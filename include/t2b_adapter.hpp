// t2b_adapter.hpp - header-only C++ adapter over the C ABI in t2b.h.
//
// Gives RELION's host code the class surface it already calls, backed by
// libt2b.so:
//   t2b::AccProjector      ~ AccProjector      (src/acc/acc_projector.h:69-78)
//   t2b::AccBackprojector  ~ AccBackprojector  (src/acc/acc_backprojector.h:51-100)
//   t2b::MlDeviceBundle    ~ MlDeviceBundle    (src/acc/cuda/cuda_ml_optimiser.h:17-72)
//   t2b::MlOptimiserCuda   ~ MlOptimiserCuda   (src/acc/cuda/cuda_ml_optimiser.h:73-186)
// Errors of the C ABI become t2b::Error exceptions, which the reference's
// thread wrapper (src/ml_optimiser.cpp:69-90) already catches per thread.
#pragma once
#include <stdexcept>
#include <string>
#include <vector>
#include "t2b.h"

namespace t2b {

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

inline void check(int rc)
{
    if (rc != T2B_OK) throw Error(rc, t2b_last_error());
}

// One context per GPU: owns projection tables, grids and the batch workspace.
class MlDeviceBundle {
public:
    explicit MlDeviceBundle(int device) { check(t2b_create(device, &ctx_)); }
    ~MlDeviceBundle() { t2b_destroy(ctx_); }
    MlDeviceBundle(const MlDeviceBundle&) = delete;
    MlDeviceBundle& operator=(const MlDeviceBundle&) = delete;
    t2b_ctx* ctx() const { return ctx_; }
    // setupTunableSizedObjects: sampling + workspace for `max_batch` particles
    void setupTunableSizedObjects(const t2b_config& cfg) { check(t2b_configure(ctx_, &cfg)); }

private:
    t2b_ctx* ctx_ = nullptr;
};

class AccProjector {
public:
    AccProjector(MlDeviceBundle& b, int iclass) : b_(b), iclass_(iclass) {}
    // returns true: the device model is (re)allocated by initMdl
    bool setMdlDim(int xdim, int ydim, int zdim, int inity, int initz, int maxr, int paddingFactor)
    {
        x_ = xdim; y_ = ydim; z_ = zdim; iy_ = inity; iz_ = initz; r_ = maxr; pad_ = paddingFactor;
        return true;
    }
    // data: interleaved complex, xdim*ydim*zdim values
    void initMdl(const float* data)
    {
        check(t2b_projector_set(b_.ctx(), iclass_, z_ > 1 ? 3 : 2, x_, y_, z_, iy_, iz_, r_, pad_, data));
    }

private:
    MlDeviceBundle& b_;
    int iclass_, x_ = 0, y_ = 0, z_ = 0, iy_ = 0, iz_ = 0, r_ = 0, pad_ = 2;
};

class AccBackprojector {
public:
    AccBackprojector(MlDeviceBundle& b, int iclass) : b_(b), iclass_(iclass) {}
    size_t setMdlDim(int xdim, int ydim, int zdim, int inity, int initz, int max_r, int paddingFactor)
    {
        x_ = xdim; y_ = ydim; z_ = zdim; iy_ = inity; iz_ = initz; r_ = max_r; pad_ = paddingFactor;
        return (size_t)xdim * ydim * zdim * 3 * sizeof(float);
    }
    void initMdl() { check(t2b_backprojector_init(b_.ctx(), iclass_, z_ > 1 ? 3 : 2, x_, y_, z_, iy_, iz_, r_, pad_)); }
    void clear() { check(t2b_backprojector_clear(b_.ctx(), iclass_)); }
    // BackProjector::enforceHermitianSymmetry on the device grid (before reconstructing)
    void enforceHermitianSymmetry() { check(t2b_backprojector_enforce_hermitian(b_.ctx(), iclass_)); }
    // BackProjector::applyPointGroupSymmetry (after enforceHermitianSymmetry); group as --sym
    void applyPointGroupSymmetry(const char* group)
    {
        check(t2b_backprojector_apply_symmetry(b_.ctx(), iclass_, group));
    }
    // BackProjector::applyHelicalSymmetry (rise in pixels; ori_size: the BackProjector's)
    void applyHelicalSymmetry(int nr_helical_asu, double helical_twist, double helical_rise, int ori_size)
    {
        check(t2b_backprojector_apply_helical(b_.ctx(), iclass_, nr_helical_asu, helical_twist, helical_rise, ori_size));
    }
    void getMdlData(float* real, float* imag, float* weight)
    {
        check(t2b_backprojector_get(b_.ctx(), iclass_, real, imag, weight));
    }
    void getMdlDataPtrs(float*& data, float*& weight)
    {
        check(t2b_backprojector_device_ptrs(b_.ctx(), iclass_, &data, &weight));
    }
    // FP64 skip-gridding division (BackProjector::reconstruct, skip_gridding)
    void reconstructDivide(double* fconv) { check(t2b_reconstruct_divide(b_.ctx(), iclass_, fconv)); }

private:
    MlDeviceBundle& b_;
    int iclass_, x_ = 0, y_ = 0, z_ = 0, iy_ = 0, iz_ = 0, r_ = 0, pad_ = 2;
};

// E-step of batches of particles on one bundle.
class MlOptimiserCuda {
public:
    explicit MlOptimiserCuda(MlDeviceBundle& b) : b_(b) {}
    // doThreadExpectationSomeParticles for one batch with host buffers; the
    // per-particle status array tells which particles hit ERRNOSIGNIFS.
    void expectationBatch(const t2b_batch& in, const t2b_result& out) { check(t2b_estep_batch_host(b_.ctx(), &in, &out)); }
    // device-resident variant; enqueued on `stream` (cudaStream_t)
    void expectationBatchDevice(const t2b_batch& in, const t2b_result& out, void* stream)
    {
        check(t2b_estep_batch_device(b_.ctx(), &in, &out, stream));
    }
    // pipelined host batches: submit returns a ticket at once (the batch's inputs copy in
    // while the previous batch computes); its buffers stay untouched until wait(ticket)
    long long submitBatch(const t2b_batch& in, const t2b_result& out)
    {
        long long t = -1;
        check(t2b_estep_submit_host(b_.ctx(), &in, &out, &t));
        return t;
    }
    void wait(long long ticket = -1) { check(t2b_estep_wait(b_.ctx(), ticket)); }

private:
    MlDeviceBundle& b_;
};

// Learned orientation proposals of one bundle (no counterpart in the reference):
// train once per iteration on particles generated from the uploaded references,
// then enable for the following batches.
class ProposalNetwork {
public:
    explicit ProposalNetwork(MlDeviceBundle& b) : b_(b) {}
    t2b_proposal_report train(const t2b_proposal_train_config& cfg)
    {
        t2b_proposal_report rep;
        check(t2b_proposal_train(b_.ctx(), &cfg, &rep));
        return rep;
    }
    void enable(int topk = 64, int rescore = 1024, int audit_every = 50, double audit_mass = 0.999)
    {
        check(t2b_proposal_enable(b_.ctx(), topk, rescore, audit_every, audit_mass));
    }
    void disable() { check(t2b_proposal_enable(b_.ctx(), 0, 0, 1, 1.0)); }

private:
    MlDeviceBundle& b_;
};

}  // namespace t2b
