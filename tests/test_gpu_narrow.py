"""The narrow phase on the device (nph_gpu_collide) against the reference's own
nph_physics_collide: each manifold the same bits (normal, point count, points, separations,
feature ids), in both orders of each pair kind, over random poses and degenerate ones, and
for two boxes resting on each other."""
from __future__ import annotations

import numpy as np
import pytest

from nepheline_b200 import abi
from tests import narrow_cases

pytestmark = pytest.mark.gpu


def live(m: np.ndarray) -> list:
    """Each manifold's normal, count and live points as bytes."""
    out = []
    for r in m:
        k = int(r["point_count"])
        out.append(r["normal"].tobytes() + r["point_count"].tobytes() + r["points"][:k].tobytes())
    return out


@pytest.mark.parametrize("kind", range(len(narrow_cases.KINDS)))
def test_closed_form_pairs_match_the_reference(ref_lib, kind):
    from nepheline_b200.solver import collide
    from oracle.refworld import ref_collide
    a, pa, b, pb, spec = narrow_cases.pairs(seed=kind)[kind]
    dev = collide(a, pa, b, pb, spec)
    ref = ref_collide(a, pa, b, pb, spec)
    assert int((ref["point_count"] > 0).sum()) > len(a) // 10
    bad = [i for i, (x, y) in enumerate(zip(live(dev), live(ref))) if x != y]
    assert not bad, (len(bad), bad[:5])


def test_stacked_boxes_match_the_reference(ref_lib):
    """Resting box contacts: face clipping reduced to four points, and GJK for boxes just apart."""
    from nepheline_b200.solver import collide
    from oracle.refworld import ref_collide
    a, pa, b, pb, spec = narrow_cases.stacked_boxes(seed=3, n=20000)
    dev = collide(a, pa, b, pb, spec)
    ref = ref_collide(a, pa, b, pb, spec)
    bad = [i for i, (x, y) in enumerate(zip(live(dev), live(ref))) if x != y]
    assert not bad, (len(bad), bad[:5])


def test_unknown_shape_types_are_refused(ref_lib):
    """A pair of an unknown type: the host-buffer call returns NPH_GPU_UNSUPPORTED, that pair
    gets the cleared manifold and every other pair its own."""
    from nepheline_b200.solver import SolverError, collide, lib
    box = np.zeros(2, abi.SHAPE_DTYPE)
    box["type"] = abi.SHAPE_BOX
    box["dims"] = 0.5
    other = box.copy()
    other["type"][1] = 7
    pose_a = np.zeros(2, abi.POSE_DTYPE)
    pose_a["rotation"][:, 3] = 1.0
    pose_b = pose_a.copy()
    pose_b["position"][:, 1] = 0.99
    spec = np.full(2, 0.04, np.float32)
    with pytest.raises(SolverError):
        collide(box, pose_a, other, pose_b, spec)
    out = np.zeros(2, abi.MANIFOLD_DTYPE)
    out["point_count"] = 99
    code = lib().nph_gpu_collide(box.ctypes.data, pose_a.ctypes.data, other.ctypes.data,
                                 pose_b.ctypes.data, spec.ctypes.data, 2, out.ctypes.data)
    assert code == abi.UNSUPPORTED
    want = collide(box[:1], pose_a[:1], other[:1], pose_b[:1], spec[:1])
    assert out[:1].tobytes() == want.tobytes() and want[0]["point_count"] == 4
    assert out[1]["point_count"] == 0 and tuple(out[1]["normal"]) == (0.0, 1.0, 0.0)


def test_async_sorted_and_unsorted_launches_agree(ref_lib):
    """nph_gpu_collide_async on device arrays: with the workspace (pairs sorted by kind on the
    device) and without (one launch) the manifolds are the same, and a pair of an unknown type
    gets the cleared manifold and is counted."""
    import torch

    from nepheline_b200 import scenes
    from nepheline_b200.solver import collide_async, collide_workspace_bytes
    a, pa, b, pb, sp = scenes.narrow_pairs(50000, seed=9)
    a["type"][123] = 9
    arrays = [a, pa, b, pb, sp]
    dev = [torch.from_numpy(np.ascontiguousarray(x).view(np.uint8).reshape(-1)).to("cuda:0") for x in arrays]
    n = len(a)
    outs = []
    for sorted_ in (False, True):
        out = torch.empty(n * abi.MANIFOLD_DTYPE.itemsize, dtype=torch.uint8, device="cuda:0")
        bad = torch.zeros(1, dtype=torch.int32, device="cuda:0")
        ws_bytes = collide_workspace_bytes(n) if sorted_ else 0
        ws = torch.empty(max(ws_bytes, 1), dtype=torch.uint8, device="cuda:0")
        collide_async(*[d.data_ptr() for d in dev], n, out.data_ptr(), bad.data_ptr(),
                      ws.data_ptr() if sorted_ else 0, ws_bytes, torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        assert int(bad.item()) == 1
        outs.append(out.cpu().numpy().view(abi.MANIFOLD_DTYPE))
    assert outs[0].tobytes() == outs[1].tobytes()
    assert outs[0][123]["point_count"] == 0 and tuple(outs[0][123]["normal"]) == (0.0, 1.0, 0.0)
    from oracle.refworld import ref_collide
    keep = np.ones(n, bool)
    keep[123] = False
    ref = ref_collide(a[keep], pa[keep], b[keep], pb[keep], sp[keep])
    got = outs[1][keep]
    bad_rows = [i for i, (x, y) in enumerate(zip(live(got), live(ref))) if x != y]
    assert not bad_rows, (len(bad_rows), bad_rows[:5])


def test_host_call_in_chunks_equals_one_launch():
    """nph_gpu_collide on host arrays, in chunks through its three streams (2, 16 and 1 chunks:
    then slots reused and arrays grown, then a small call), gives the bits of one unsorted
    launch over all the pairs; from page-locked and from ordinary host memory alike."""
    import torch

    from nepheline_b200 import scenes
    from nepheline_b200.solver import collide, collide_async, collide_host, collide_release

    def one_launch(arrays, n):
        dev = [torch.from_numpy(np.ascontiguousarray(x).view(np.uint8).reshape(-1)).to("cuda:0")
               for x in arrays]
        out = torch.empty(n * abi.MANIFOLD_DTYPE.itemsize, dtype=torch.uint8, device="cuda:0")
        collide_async(*[d.data_ptr() for d in dev], n, out.data_ptr(), 0, 0, 0,
                      torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        return out.cpu().numpy().view(abi.MANIFOLD_DTYPE)

    for n, seed in ((131072, 3), (16 * 65536 + 4 * 65536 + 777, 4), (1000, 5)):
        arrays = scenes.narrow_pairs(n, seed=seed)
        want = one_launch(arrays, n)
        got = collide(*arrays)
        assert got.tobytes() == want.tobytes(), n
        host = [torch.from_numpy(np.ascontiguousarray(x).view(np.uint8).reshape(-1)).pin_memory()
                for x in arrays]
        out = torch.zeros(n * abi.MANIFOLD_DTYPE.itemsize, dtype=torch.uint8).pin_memory()
        collide_host(*[h.data_ptr() for h in host], n, out.data_ptr())
        assert out.numpy().tobytes() == want.tobytes(), n
    # Released, then made again by the next call.
    collide_release()
    collide_release()
    assert collide(*arrays).tobytes() == want.tobytes()


def test_host_call_edge_counts():
    """No pairs: nothing to do; one pair: the one-launch result."""
    from nepheline_b200 import scenes
    from nepheline_b200.solver import collide, collide_host
    a, pa, b, pb, sp = scenes.narrow_pairs(3, seed=6)
    assert len(collide(a[:0], pa[:0], b[:0], pb[:0], sp[:0])) == 0
    collide_host(0, 0, 0, 0, 0, 0, 0)
    one = collide(a[:1], pa[:1], b[:1], pb[:1], sp[:1])
    three = collide(a, pa, b, pb, sp)
    assert one.tobytes() == three[:1].tobytes()
