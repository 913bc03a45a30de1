// NCCL entry points of the decomposed dycore, resolved at run time.
//
// The library does not link NCCL: a single-GPU process never needs it, and a
// process that already holds NCCL (PyTorch ships its own libnccl.so.2) must
// not load a second copy.  pu::nccl() opens "libnccl.so.2" on first use --
// the loader returns the copy already in the process if there is one -- and
// resolves the handful of calls the halo exchange and the profile sums use.
// Types and enums come from the NCCL header, whose C ABI is stable.
#pragma once

#include <nccl.h>

#include <string>

namespace pu {

struct NcclApi {
  bool ok = false;
  std::string error;  // why loading failed
  ncclResult_t (*GetUniqueId)(ncclUniqueId *) = nullptr;
  ncclResult_t (*CommInitRank)(ncclComm_t *, int, ncclUniqueId, int) = nullptr;
  ncclResult_t (*CommDestroy)(ncclComm_t) = nullptr;
  ncclResult_t (*GroupStart)() = nullptr;
  ncclResult_t (*GroupEnd)() = nullptr;
  ncclResult_t (*Send)(const void *, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
  ncclResult_t (*Recv)(void *, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
  ncclResult_t (*AllReduce)(const void *, void *, size_t, ncclDataType_t, ncclRedOp_t, ncclComm_t,
                            cudaStream_t) = nullptr;
  ncclResult_t (*AllGather)(const void *, void *, size_t, ncclDataType_t, ncclComm_t, cudaStream_t) = nullptr;
  const char *(*GetErrorString)(ncclResult_t) = nullptr;
};

// The process-wide table (loaded once, thread-safe); check .ok before use.
NcclApi &nccl();

}  // namespace pu
