"""The recorded reference driver trace and its replay harness, on the CPU.

Replaying the reference's recorded backend calls into the oracle's
NumpyBackend (complex128, the reference's arithmetic) reproduces every
recorded result and amplitude (to the 10 digits the trace keeps), so the GPU replay in ``test_gpu_dropin.py``
tests the backend and not the harness."""
import numpy as np

import dropin_replay
import qtensor_port as port


def test_trace_replays_exactly_on_the_oracle_backend():
    w = dropin_replay.load()
    for name in ('cfg1', 'cfg2'):
        for rec in w[name]['edges']:
            def check(k, res, rec=rec):
                call = rec['calls'][k]
                assert res.name == call['name']
                assert [dropin_replay.var_rec(v) for v in res.indices] == call['indices']
                got = np.asarray(res.data, dtype=np.complex128).reshape(-1)
                if 'data' in call:
                    assert np.allclose(got, [complex(*z) for z in call['data']], atol=1e-7)
                else:
                    assert abs(got.sum() - complex(*call['sum'][0])) < 1e-7 * max(1.0, call['norm2'])
            amp, _ = dropin_replay.replay_edge(port.NumpyBackend(), rec, check=check)
            assert np.allclose(amp, [complex(*z) for z in rec['amplitude']], atol=1e-7)


def test_trace_covers_the_whole_cfg1_energy():
    from conftest import golden
    w = dropin_replay.load()['cfg1']
    ref = golden()['cfg1_default']
    assert [r['edge'] for r in w['edges']] == ref['edges']
    total = sum(complex(*r['amplitude'][0]) for r in w['edges'])
    assert abs((len(ref['edges']) - total.real) / 2 - ref['energy']) < 1e-9
