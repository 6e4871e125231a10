#ifndef MOSP_B200_DEVICE_GRAPH_CUH
#define MOSP_B200_DEVICE_GRAPH_CUH

// Multi-objective graph resident on the GPU (same interface as the
// reference, SMShovan/MOSP-CUDA headers/deviceGraph.cuh:16-37): out- and
// in-edge CSR with one contiguous weight column per objective.

#include "deviceArray.cuh"
#include "sospUpdateGpu.cuh"

struct CsrGraph;

struct DeviceGraph {
  int numberOfNodes = 0;
  int numberOfEdges = 0;
  int numberOfObjectives = 0;
  DeviceArray<int> outRowPtr, outColInd, outWeights; ///< weights: K columns
  DeviceArray<int> inRowPtr, inColInd, inWeights;    ///< reverse graph

  /// Out-edge view of objective k.
  DeviceCsr out(int k) const;
  /// In-edge view of objective k.
  DeviceCsr in(int k) const;
};

/// Upload the out-edge CSR once; the weight columns and the reverse CSR
/// are built on the GPU (mosp_build_device_graph), which also checks the
/// CSR.
bool uploadDeviceGraph(const CsrGraph &graph, DeviceGraph &device);

#endif // MOSP_B200_DEVICE_GRAPH_CUH
