// Fast-mode CPIC transfers: the grid update (compatible and incompatible
// fields) and the per-block G2P + particle update of nxm_transfer.inc.cuh,
// built with the fast arithmetic (multiply-adds may fuse, the fast model
// forms) and the CPIC branches.  A particle without affinity bits takes the
// factored gather of the plain fast path; one with affinity takes the per-node
// gather that substitutes incompatible nodes (solver/g2p.rs:206-257).  The
// scatter P2G of this mode is k_p2g<true> (nxm_transfer_fast.cu).
#define NXM_NS fast_cpic
#define NXM_FAST true
#define NXM_CPIC 1
#include "nxm_transfer.inc.cuh"
