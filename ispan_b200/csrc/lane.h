// lane.h -- internal interface between the request server (server.cu) and
// the contexts of pipeline.cu.  Not part of the C ABI.
//
// A server lane is a context whose device scratch and union buffers are not
// allocated with cudaMalloc but carved, batch by batch, out of a region of
// the server's device-memory budget (cudaMalloc and cudaFree synchronise the
// whole device, which would stall the other lanes' work).  Its persistent
// stage kernels are sized for a share of the SMs, so the persistent kernels
// of all lanes are co-resident whatever mix of them runs at once.
#pragma once
#include <cstddef>
#include <cstdint>

#include "../../include/ispan_b200.h"

// device bytes a lane needs for a batch of n graphs with V vertices and E
// edges in total, V_host of the vertices in host-resident graphs (whose
// offsets are staged on the device): every scratch array, the union CSR and
// its tables
size_t lane_region_bytes(int64_t V, int64_t E, int64_t n, int64_t V_host);
// carve the batch's arrays out of [base, base + bytes); the lane is then
// ready for ispan_graphs_pack / ispan_graphs_run of that batch
int lane_bind(ispan_ctx *c, void *base, size_t bytes, int64_t V, int64_t E, int64_t n, int64_t V_host);
// the region is handed back (the caller frees it in its budget)
void lane_unbind(ispan_ctx *c);
// persistent grids sized for nsm SMs
int lane_set_sm_share(ispan_ctx *c, int nsm);
// pinned host tables for batches of up to n graphs, allocated once
int lane_reserve_host(ispan_ctx *c, int64_t n);
