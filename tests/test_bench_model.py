"""The algorithmic-bytes model behind bench.py's roofline figure
(algorithmic_bytes, segment_record_bytes) on a case counted by hand: visited
pairs, neighbour records, contributing pairs and the segment records of the
visited pairs (hit pixels, non-empty intervals, pairs left without records)."""

import types

import torch

import bench


def _ids(tn_id, tf_id):
    return (tn_id + 2) | ((tf_id + 2) << 16)


def test_algorithmic_bytes_counted_by_hand():
    bins = types.SimpleNamespace(tile_offsets=torch.tensor([0, 3, 5]), tile_prims=torch.tensor([0, 1, 2, 1, 3],
                                 dtype=torch.int32), n_pairs=5)
    ao = torch.tensor([0, 1, 3, 6, 10], dtype=torch.int32)  # degrees 1, 2, 3, 4
    # tile width 8: two warps per (pair); masks and record offsets per (pair, warp)
    mask = torch.tensor([[0b11, 0], [0b1, 0b101], [0b1111, 0], [0, 0b1], [0b1, 0]], dtype=torch.int32)
    offs = torch.tensor([[0, -1], [2, 3], [5, -1], [-1, -1], [9, -1]], dtype=torch.int32)
    cap = 16
    seg = torch.zeros((cap * 4, 4), dtype=torch.float32)
    rec = {0: (0.1, 0.5, _ids(-1, 0)), 1: (0.5, 0.2, _ids(-1, -1)), 2: (0.2, 0.3, _ids(-1, -1)),
           3: (0.3, 0.9, _ids(3, -1)), 4: (0.9, 0.9, _ids(-1, -1)), 9: (0.0, 1.0, _ids(-1, -1))}
    view = seg.view(cap, 4, 4)
    for i, (tn, tf, ids) in rec.items():
        view[i, 0, 0], view[i, 0, 1] = tn, tf
        view[i, 0, 2] = torch.tensor([ids], dtype=torch.int32).view(torch.float32)[0]
    stats = dict(bins=bins, early_stop=torch.tensor([2, 2], dtype=torch.int32), adjacency_offsets=ao,
                 contrib_pairs=torch.tensor([1, 2], dtype=torch.int32), n_prims=4, tile_width=8,
                 segments=(seg, mask.flatten(), offs.flatten(), torch.tensor([7]), 5, cap, True))
    st = bench.algorithmic_bytes(stats, 8, 8)
    # visited: pairs 0, 1 of tile 0 and 3, 4 of tile 1 -> prims 0, 1, 1, 3 -> degree 1 + 2 + 2 + 4
    assert (st["V"], st["U"], st["deg"], st["pairs"], st["T"]) == (4, 3, 9, 5, 2)
    r = st["records"]
    # hits with records: 2 + 1 + 2 + 1 (pair 3's hit found the buffer full); non-empty: records 0, 2, 3, 9;
    # a power face bounds records 0 and 3
    assert (r["hit_pixels"], r["nonempty_pixels"], r["face_bounded_pixels"], r["clipped_again_pairs"]) == (6, 4, 2, 1)
    assert r["bytes"] == 8 * 4 * 2 + 16 * 6 + 48 * 4
    fwd = 256 * 4 + 8 * 9 + 4 * 4 + 8 * 3 + 32 * 64 + 4 * 4
    bwd = 256 * 4 + 8 * 9 + 4 * 4 + 36 * 64 + 2 * 256 * 3
    assert st["fwd"] == fwd + r["bytes"]
    assert st["bwd"] == bwd + r["bytes"] - 8 * 9
    # intervals only: no plane part
    stats["segments"] = (seg.view(cap, 4, 4)[:, 0].contiguous(), mask.flatten(), offs.flatten(), torch.tensor([7]), 5,
                         cap, False)
    assert bench.algorithmic_bytes(stats, 8, 8)["records"]["bytes"] == 8 * 4 * 2 + 16 * 6
