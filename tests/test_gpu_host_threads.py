"""GPU: the host-buffer entry points from several host threads at once.

Pageable host buffers (the drop-in classes' storage) are staged through a pinned
ring per host thread and device, filled and drained by one shared pool of copy
threads. Four Python threads encode and decode different textures concurrently
through the drop-in API (the GIL is released during each call); every result
must equal the same call made alone, and the decodes must equal the oracle's.
"""

import threading

import numpy as np
import pytest

import quicktex_b200 as qt
import workloads as syn
from quicktex_b200.s3tc.bc1 import BC1Decoder, BC1Encoder
from quicktex_b200.s3tc.bc3 import BC3Encoder
from quicktex_b200.s3tc.bc5 import BC5Encoder

pytestmark = pytest.mark.gpu


def _cases():
    out = []
    for k, (w, h) in enumerate(((1536, 1024), (1030, 770), (2048, 2048), (517, 1999))):
        img = syn.alpha_mix(w, h, workload=12, stream=k)
        out.append((qt.RawTexture.frombytes(img.tobytes(), w, h), w, h))
    return out


def _work(tex, k):
    enc = [BC1Encoder(5), BC3Encoder(3), BC5Encoder(0, 1), BC1Encoder(10, BC1Encoder.ColorMode.ThreeColor)][k % 4]
    blocks = enc.encode(tex)
    dec = BC1Decoder(True).decode(blocks) if isinstance(enc, BC1Encoder) else None
    return blocks.tobytes(), (dec.tobytes() if dec is not None else b"")


def test_concurrent_host_calls_match_sequential(oracle_lib):
    cases = _cases()
    alone = [_work(t, k) for k, (t, _, _) in enumerate(cases)]
    results = [[None] * len(cases) for _ in range(3)]
    errors = []

    def run(rep):
        try:
            for k, (t, _, _) in enumerate(cases):
                j = (k + rep) % len(cases)  # threads start on different textures
                results[rep][j] = _work(cases[j][0], j)
        except Exception as e:  # surfaced below
            errors.append(e)

    threads = [threading.Thread(target=run, args=(r,)) for r in range(3)]
    for t in threads:
        t.start()
    extra = [_work(t, k) for k, (t, _, _) in enumerate(cases)]  # the main thread as a fourth caller
    for t in threads:
        t.join()
    assert not errors, errors
    for r in results + [extra]:
        assert r == alone
    for k, (t, w, h) in enumerate(cases):
        if k % 4 in (0, 3):
            blocks = np.frombuffer(alone[k][0], np.uint8)
            assert alone[k][1] == oracle_lib.bc1_decode(blocks, w, h, 0, True)
