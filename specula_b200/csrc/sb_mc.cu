// Monte-Carlo step over geometry groups: the plan and the C ABI.  The stages
// live beside the kernels they reuse (sb_atmo.cu, sb_sh.cu, sb_detector.cu,
// sb_control.cu); this file carves the workspace, has each stage build its
// arguments once, and issues the six launches of a step.
#include <new>

#include "sb_mc.cuh"

struct sb_mc_handle {
    int n_groups;
    sb::McBlob atmo, sh, chain, rec, dm;
};

namespace {

int check_groups(const char *who, const sb_mc_group *gs, int n) {
    if (!gs || n < 1 || n > SB_MC_MAX_GROUPS)
        return sb::fail(SB_EINVAL, "%s: 1 to %d groups", who, SB_MC_MAX_GROUPS);
    for (int g = 0; g < n; ++g)
        if (gs[g].n_batch < 1) return sb::fail(SB_EINVAL, "%s: group %d has no realisations", who, g);
    return SB_OK;
}

// workspace of each stage, in the order they are carved
void stage_bytes(const sb_mc_group *gs, int n, size_t b[4]) {
    b[0] = sb::mc_atmo_workspace(gs, n);
    b[1] = sb::mc_sh_workspace(gs, n);
    b[2] = sb::mc_chain_workspace(gs, n);
    b[3] = sb::mc_control_workspace(gs, n);
}

}  // namespace

extern "C" size_t sb_mc_workspace_bytes(const sb_mc_group *groups, int n_groups) {
    sb::clear_error();
    if (check_groups("sb_mc_workspace_bytes", groups, n_groups)) return 0;
    size_t b[4];
    stage_bytes(groups, n_groups, b);
    return b[0] + b[1] + b[2] + b[3] + 256;
}

extern "C" int sb_mc_create(const sb_mc_group *groups, int n_groups, void *workspace, size_t workspace_bytes,
                            sb_mc_handle **handle, void *stream) {
    sb::clear_error();
    const char *who = "sb_mc_create";
    int rc = check_groups(who, groups, n_groups);
    if (rc) return rc;
    if (!handle) return sb::fail(SB_EINVAL, "%s: null handle pointer", who);
    *handle = nullptr;
    const size_t need = sb_mc_workspace_bytes(groups, n_groups);
    if (!workspace || (uintptr_t)workspace % 256 || workspace_bytes < need)
        return sb::fail(SB_ESCRATCH, "%s: workspace needs %zu bytes, 256-byte aligned", who, need);
    size_t b[4];
    stage_bytes(groups, n_groups, b);
    unsigned char *w = static_cast<unsigned char *>(workspace);
    sb_mc_handle *h = new (std::nothrow) sb_mc_handle();
    if (!h) return sb::fail(SB_ECUDA, "%s: out of host memory", who);
    h->n_groups = n_groups;
    cudaStream_t st = sb::as_stream(stream);
    sb::McShParts parts = {};
    rc = sb::mc_atmo_prepare(groups, n_groups, w, h->atmo, st);
    if (!rc) rc = sb::mc_sh_prepare(groups, n_groups, w + b[0], h->sh, parts);
    if (!rc) rc = sb::mc_chain_prepare(groups, n_groups, parts, w + b[0] + b[1], h->chain);
    if (!rc) rc = sb::mc_control_prepare(groups, n_groups, w + b[0] + b[1] + b[2], h->rec, h->dm, st);
    if (rc) {
        delete h;
        return rc;
    }
    *handle = h;
    return SB_OK;
}

extern "C" int sb_mc_step(const sb_mc_handle *h, void *stream) {
    sb::clear_error();
    if (!h) return sb::fail(SB_EINVAL, "sb_mc_step: null handle");
    cudaStream_t st = sb::as_stream(stream);
    int rc = sb::mc_atmo_launch(h->atmo, 0, st);
    if (!rc) rc = sb::mc_sh_launch(h->sh, st);
    if (!rc) rc = sb::mc_chain_launch(h->chain, st);
    if (!rc) rc = sb::mc_rec_launch(h->rec, st);
    if (!rc) rc = sb::mc_dm_launch(h->dm, 0, 0, st);
    return rc;
}

extern "C" int sb_mc_stage(const sb_mc_handle *h, int stage, int parity, void *stream) {
    sb::clear_error();
    if (!h) return sb::fail(SB_EINVAL, "sb_mc_stage: null handle");
    if (parity < -1 || parity > 1) return sb::fail(SB_EINVAL, "sb_mc_stage: parity must be -1, 0 or 1");
    cudaStream_t st = sb::as_stream(stream);
    switch (stage) {
        case SB_MC_ATMO: return sb::mc_atmo_launch(h->atmo, parity < 0 ? 0 : parity ^ 1, st);
        case SB_MC_SH: return sb::mc_sh_launch(h->sh, st);
        case SB_MC_CHAIN: return sb::mc_chain_launch(h->chain, st);
        case SB_MC_REC: return sb::mc_rec_launch(h->rec, st);
        case SB_MC_DM: return parity < 0 ? sb::mc_dm_launch(h->dm, 0, 0, st) : sb::mc_dm_launch(h->dm, 1, parity, st);
        default: return sb::fail(SB_EINVAL, "sb_mc_stage: no stage %d", stage);
    }
}

extern "C" void sb_mc_destroy(sb_mc_handle *h) { delete h; }
