// C ABI of the batched commit (included at the end of pil2_b200.cu: uses its error helpers).
#pragma once
#include "batch.cuh"

static int batch_insts(const B200BatchInstance *in, uint64_t n, std::vector<batch::Inst> &out)
{
    out.clear();
    for (uint64_t i = 0; i < n; i++) {
        const B200BatchInstance &x = in[i];
        int rc = check_shape(x.nBits, x.nBitsExt, x.nCols, x.arity);
        if (rc) return rc;
        if (!x.d_tree || (x.nCols && (!x.d_trace || !x.d_scratch || !x.d_lde)))
            return set_err(B200_EINVAL, "batch instance " + std::to_string(i) + ": null buffer");
        out.push_back(batch::Inst{x.d_trace, x.d_scratch, x.d_lde, x.d_tree, (uint32_t)x.nBits, (uint32_t)x.nBitsExt,
                                  (uint32_t)x.nCols, (uint32_t)x.arity});
    }
    return B200_OK;
}

static int batch_kernel_attrs()
{
    static bool done[64];
    int dev = 0;
    CK(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev < 0 || dev >= 64) return set_err(B200_EINVAL, "device index out of range");
    if (!done[dev]) {
        CK(cudaFuncSetAttribute(batch::pass_grouped, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (NTT_TILE_MAX + NTT_TILE_MAX / 16) * 8),
           "pass_grouped smem attribute");
        CK(batch::set_grouped_fixed_attrs(), "pass_fixed_grouped smem attributes");
        done[dev] = true;
    }
    return B200_OK;
}

extern "C" void *b200_batch_plan_new(const B200BatchInstance *inst, uint64_t n)
{
    if (!inst || n == 0) {
        set_err(B200_EINVAL, "b200_batch_plan_new: empty batch");
        return nullptr;
    }
    if (ensure_init_current() || batch_kernel_attrs()) return nullptr;
    std::vector<batch::Inst> v;
    if (batch_insts(inst, n, v)) return nullptr;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    auto *plan = new batch::Plan();
    if (!plan->build(v, sms, g_native_family.load())) {
        delete plan;
        set_err(B200_EINVAL, "b200_batch_plan_new: unsupported shape");
        return nullptr;
    }
    cudaError_t e = plan->upload();
    if (e != cudaSuccess) {
        delete plan;
        cuda_err(e, "b200_batch_plan_new upload");
        return nullptr;
    }
    return plan;
}

extern "C" int b200_batch_plan_run(void *plan_, uint64_t *roots_host, void *stream, int use_graph)
{
    auto *plan = (batch::Plan *)plan_;
    if (!plan) return set_err(B200_EINVAL, "null plan");
    if (use_graph && !stream) return set_err(B200_EINVAL, "graph replay needs a created stream");
    cudaStream_t s = (cudaStream_t)stream;
    CK(plan->run(s, use_graph != 0), "batch run");
    if (roots_host) {
        CK(cudaStreamSynchronize(s), "batch sync");
        memcpy(roots_host, plan->h_roots, 32 * plan->inst.size());
    }
    return B200_OK;
}

extern "C" void b200_batch_plan_free(void *plan) { delete (batch::Plan *)plan; }

extern "C" uint64_t b200_batch_plan_launches(void *plan_)
{
    auto *plan = (batch::Plan *)plan_;
    return plan ? plan->launches.size() + 1 : 0;
}

extern "C" int b200_commit_batch_device(const B200BatchInstance *inst, uint64_t n, uint64_t *roots_host,
                                        void *stream)
{
    void *plan = b200_batch_plan_new(inst, n);
    if (!plan) return B200_EINVAL;
    int rc = b200_batch_plan_run(plan, roots_host, stream, 0);
    if (!rc && !roots_host) {
        cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
        if (e != cudaSuccess) rc = cuda_err(e, "batch sync");
    }
    b200_batch_plan_free(plan);
    return rc;
}
