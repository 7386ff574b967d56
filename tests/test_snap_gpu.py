"""Standalone snapshot store (rtm_snap call sequence, snap_helpers/rtm_snap.h:
19-41): snapshots written on a "forward" stream come back last-in first-out,
bit for bit, from the device tier and from the pinned host tier."""
import numpy as np
import pytest

import miniappsforhpe_b200 as P


@pytest.mark.gpu
@pytest.mark.parametrize("dev_cap,host_cap", [(6, 0), (2, 4), (0, 3)], ids=["device", "tiered", "host"])
def test_lifo_round_trip(dev_cap, host_cap):
    import torch

    n = dev_cap + host_cap
    sizes = [3000, 1234, 777]
    st = torch.cuda.Stream()
    g = torch.Generator(device="cuda").manual_seed(n)
    store = P.SnapshotStore(sizes, dev_cap, host_cap)
    vols = [torch.empty(k, device="cuda") for k in sizes]
    written = []
    with torch.cuda.stream(st):
        for i in range(n):
            store.lock_for_write()
            for v in vols:  # the "forward step" overwrites the volumes on the stream
                v.copy_(torch.randn(v.numel(), device="cuda", generator=g))
            written.append([v.cpu().numpy() for v in vols])
            store.start_write(vols, st.cuda_stream)
        assert store.count() == n
        with pytest.raises(P.TTIError):  # full
            store.start_write(vols, st.cuda_stream)
        out = [torch.zeros(k, device="cuda") for k in sizes]
        for i in reversed(range(n)):
            store.start_read(out, st.cuda_stream)
            store.finish_read(st.cuda_stream)
            got = [o.cpu().numpy() for o in out]
            for a, b in zip(got, written[i]):
                np.testing.assert_array_equal(a, b)
        assert store.count() == 0
        with pytest.raises(P.TTIError):  # empty
            store.start_read(out, st.cuda_stream)
    store.close()
