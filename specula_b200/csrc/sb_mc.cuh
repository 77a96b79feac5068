// Monte-Carlo step over geometry groups: the interface between the stage
// implementations (each in the file of the kernels it reuses) and the plan in
// sb_mc.cu.  A stage's prepare function validates the groups, copies its
// tables into its share of the workspace and writes its kernel arguments
// and grids into a blob; its launch function issues the stage from the blob.
#pragma once
#include "sb_common.cuh"

namespace sb {

constexpr int kMcMaxGroups = SB_MC_MAX_GROUPS;

// kernel arguments and grid of one stage (each stage's arguments stay below
// the 4 KB a kernel parameter block has always been allowed)
struct alignas(128) McBlob {
    unsigned char b[8192];
};

// the SH stage's per-CTA partial sums, read by the detector stage
struct McShParts {
    const float *part_I[kMcMaxGroups];   // [n_batch][nparts]
    const float *part_A[kMcMaxGroups];
    int nparts[kMcMaxGroups];
};

inline size_t mc_align(size_t b) { return (b + 255) & ~(size_t)255; }

// stages 1-2: layer parameters, then layers and the on-axis field in one
// launch (a group of more than 16 layers: layers and field separately); the
// field takes mirror-phase buffer sel (0: dm_phase, 1: dm_phase_alt)
size_t mc_atmo_workspace(const sb_mc_group *g, int n);
int mc_atmo_prepare(const sb_mc_group *g, int n, void *ws, McBlob &blob, cudaStream_t st);
int mc_atmo_launch(const McBlob &blob, int sel, cudaStream_t st);

// stage 3: SH forward (one launch)
size_t mc_sh_workspace(const sb_mc_group *g, int n);
int mc_sh_prepare(const sb_mc_group *g, int n, void *ws, McBlob &blob, McShParts &parts);
int mc_sh_launch(const McBlob &blob, cudaStream_t st);

// stage 4: normalisation, detector, slopes (one launch)
size_t mc_chain_workspace(const sb_mc_group *g, int n);
int mc_chain_prepare(const sb_mc_group *g, int n, const McShParts &parts, void *ws, McBlob &blob);
int mc_chain_launch(const McBlob &blob, cudaStream_t st);

// stages 5-6: reconstructor + integrators, mirror (two launches)
size_t mc_control_workspace(const sb_mc_group *g, int n);
int mc_control_prepare(const sb_mc_group *g, int n, void *ws, McBlob &rec, McBlob &dm, cudaStream_t st);
int mc_rec_launch(const McBlob &blob, cudaStream_t st);
// mirror from commands (cmd 0) or commands_next (1) into buffer sel
int mc_dm_launch(const McBlob &blob, int cmd, int sel, cudaStream_t st);

}  // namespace sb
