// Host-side description of one work-list closure (closure_rounds.cu), shared by the
// context code that fills it.
#pragma once
#include "c3d_common.cuh"

#include <cstddef>
#include <mutex>
#include <vector>

namespace c3d {

struct RoundsLaunch {
    const ClosureParams *P;
    const double *chunks;      // direct: (NMP+1) x QCP chunks; Gaunt: (NM2P+1) x QCP chunks
    int nm2;                   // Gaunt: extended moments (chunk rows: nm2 + the weight row)
    const GauntTerm *gstream;  // Gaunt: assembly streams, entry s of thread t at s*128 + t
    int streamLen;             // entries per thread
    double m0;                 // M[0][0]
    long long ncells;
    const int *cellMap;        // closure cell i -> grid cell cellMap[i] (null: identity)
    double *u, *alpha;
    int *iters, *iterGamma, *regIdx, *status;
    unsigned long long *failCount, *stats;
    double *gamma, *normG;     // per-cell final gamma and |g| (may be null)
    float *cond;               // per-cell condition estimate records (may be null)
    void *state;               // ncells x rounds_state_bytes(nm)
    int *listA, *listB;        // NLISTS x ncells each (one list per precision level)
    unsigned int *counts;      // 2 NLISTS device counters
    unsigned int *hostCount;   // NLISTS pinned
    double *buf;               // batch x rounds_buf_doubles doubles
    long long batch;           // list entries per pass/Newton launch pair
    // mixed precision (P->mixed): FP64 rows (nm rows of M2 + weights) and the A operand
    // chunks of each format (BF16; TF32 hi then lo)
    const double *mixF64;
    const unsigned char *mixA[2];
    // probe of first visits (P->probe): the Gaunt terms of H's column 0, g0n per row (col -2:
    // padding), for the FP64 closure's gradient
    const GauntTerm *g0;
    int g0n;
    int *errorFlag;
    cudaStream_t stream;
    long long *launches;
    long long *hostSyncs; // host-driven rounds: one wait per round
    long long maxRounds;
    // ansatz hand-off to the kinetic flux (null psi: none): psi[q psiNall + c] of every cell
    // the probe solves, and the list (with its device count) of cells whose psi is rewritten
    // after the closure
    double *psi;
    long long psiNall;
    int *refresh;
    unsigned int *refreshCount;
    // device flag: psi holds every non-face-ghost cell's ansatz for the starting multipliers
    // (the probe then writes only face ghosts); gnx..gnz the grid's interior sizes
    const int *psiValid;
    int gnx, gny, gnz;
    // graph-resident round loop (rounds_graph_new; null: host-driven rounds) and the device
    // counter of the kernels its loop launches
    void *graphs;
    unsigned long long *launchDev;
    // capture into an RK stage's graph (null: launch): the closure is appended to the graph
    // being captured on captureStreams[0], whose top-level graph is captureTop;
    // captureStreams[1], [2] capture the loop and switch bodies
    cudaGraph_t captureTop;
    cudaStream_t *captureStreams;
};

cudaError_t launch_closure_rounds(const RoundsLaunch &R, bool gaunt);
size_t rounds_state_bytes(int nm);
size_t rounds_buf_doubles(int nm, int nm2, bool gaunt, bool mixed);
size_t mixed_a_chunk_bytes(int nm2, int fmt);
bool rounds_gaunt_supported(int nm);
void *rounds_graph_new();
std::mutex &graph_build_mutex(); // held while a graph is captured and instantiated
// Appends a conditional node (WHILE, IF or SWITCH with size bodies) after the current
// dependencies of the graph being captured on st; *bodies receives its body graphs.
cudaError_t capture_conditional(cudaStream_t st, cudaGraphConditionalHandle h,
                                cudaGraphConditionalNodeType type, unsigned int size,
                                cudaGraph_t **bodies);
void rounds_graph_free(void *g);
// What a captured closure depends on (options, sizes, buffers): equal keys, same graph.
std::vector<unsigned char> rounds_graph_key(const RoundsLaunch &R, bool gaunt);

} // namespace c3d
