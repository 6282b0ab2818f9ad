"""The traversal operator headers (include/operators.cuh, load_balance.cuh, algs.cuh) compile
for sm_100a in a user's translation unit, with every call form the reference's algorithms use
(include/operators.cuh in the reference): vertex operators over the graph or an array or the
load balancer's array; edge operators over the graph, a vertex array, a frontier queue, the load
balancer's array and a batch; a device queue appended from a kernel. Build only (no GPU needed);
tests/test_ref_ops_gpu.py runs the reference's algorithms on them."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"

SRC = r'''
#include "cuStinger.hpp"
#include "operators.cuh"

using namespace cuStingerAlgs;

struct Meta {
  vertexQueue q;
  int* level;
  unsigned long long* sum;
};

struct Ops {
  static __device__ void init(cuStinger* cs, vertexId_t v, void* m) { ((Meta*)m)->level[v] = cs->getMaxNV(); }
  static __device__ void visit(cuStinger* cs, vertexId_t s, vertexId_t d, void* m) {
    Meta* md = (Meta*)m;
    if (atomicCAS(md->level + d, cs->getMaxNV(), 1) == cs->getMaxNV()) md->q.enqueue(d);
    atomicAdd(md->sum, (unsigned long long)(s + d));
  }
};

void run(cuStinger& cs, BatchUpdate& bu, vertexId_t* arr, length_t len) {
  Meta h;
  h.q.Init(cs.nv);
  Meta* d = (Meta*)allocDeviceArray(1, sizeof(Meta));
  copyArrayHostToDevice(&h, d, 1, sizeof(Meta));
  cusLoadBalance all(cs), nonzero(cs, false, true), sized(cs.nv);
  allVinG_TraverseVertices<Ops::init>(cs, d);
  allVinA_TraverseVertices<Ops::init>(cs, d, arr, len);
  allVinA_TraverseVertices<Ops::init>(cs, d, all);
  allEinG_TraverseEdges<Ops::visit>(cs, d);
  allVinA_TraverseEdges<Ops::visit>(cs, d, arr, len);
  allVinA_TraverseEdges_LB<Ops::visit>(cs, d, sized, h.q);
  allVinA_TraverseEdges_LB<Ops::visit>(cs, d, nonzero);
  allEinA_TraverseEdges<Ops::visit>(cs, d, bu);
  copyArrayDeviceToHost(d, &h, 1, sizeof(Meta));
  vertexQueue other(8);
  vertexQueue::swapQueues(&h.q, &other);
  freeDeviceArray(d);
}
'''


@pytest.mark.skipif(not os.path.exists(NVCC), reason="no nvcc")
def test_operator_headers_compile(tmp_path):
    src = tmp_path / "ops_user.cu"
    src.write_text(SRC)
    r = subprocess.run([NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "-c", "-I",
                        os.path.join(ROOT, "include"), str(src), "-o", str(tmp_path / "ops_user.o")],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]


def test_every_reference_algorithm_compiles_on_these_headers():
    """The reference's BFS, connected components, PageRank, betweenness centrality and static and
    streaming Katz sources (its src/ tree) compile unmodified against include/ (oracle/Makefile
    target algs_check; skipped where the reference tree is absent)."""
    from oracle import make_args
    r = subprocess.run(["make", "-s", "-f", os.path.join(ROOT, "oracle", "Makefile"), "algs_check"] + make_args(),
                       capture_output=True, text=True, timeout=900)
    if "reference not present" in r.stdout:
        pytest.skip("reference tree absent")
    assert r.returncode == 0 and "all reference algorithms compile" in r.stdout, r.stdout[-3000:] + r.stderr[-3000:]
