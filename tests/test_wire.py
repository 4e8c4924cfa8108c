"""Wire formats: circuits round-trip through bytes with their handles and
levels intact, malformed blobs are rejected (CPU); device-form keys export
and import without conversion, giving the same gate words, and a blob from
another NTT root or parameter set is refused (GPU)."""
import numpy as np
import pytest

from conftest import oracle, oracle_setup, pz


def mixed_circuit():
    P = pz()
    C = P.Circuit()
    a, b = C.input_u8(), C.input_u8()
    s = C.input()
    C.outputs(C.u8_add(a, b))
    q, r, f = C.u8_div_rem(a, b)
    C.outputs(q)
    C.output(f)
    C.output(C.not_(C.gate("xnor", a[0], s)))
    C.outputs(C.u8_mux(a, b, s))
    return C


def test_circuit_round_trip():
    P = pz()
    C = mixed_circuit()
    blob = C.serialize()
    D = P.Circuit.deserialize(blob)
    assert D.serialize() == blob
    assert D.info() == C.info() and D.level_sizes() == C.level_sizes()
    assert (D.n_inputs, D.n_outputs) == (C.n_inputs, C.n_outputs)
    # the deserialized circuit schedules identically in the executor
    S = P.Server(device=P.DRY_RUN, arena_bytes=1 << 26, max_items=4096)
    sid = S.add_virtual_session(P.param_id("NI_8P"))
    j1, j2 = S.submit(sid, C), S.submit(sid, D)
    per_step = []
    while S.stats()["active"] or S.stats()["pending"]:
        per_step.append(S.step())
    sizes = C.level_sizes()
    assert per_step == [2 * x for x in sizes]
    assert S.status(j1)["state"] == S.status(j2)["state"] == 2


def test_malformed_circuit_blobs_rejected():
    P = pz()
    blob = bytearray(mixed_circuit().serialize())
    bad = [bytes(blob[:10]), bytes(blob[:-4]), b"\x00" * len(blob),
           bytes(np.random.default_rng(1).integers(0, 256, len(blob), dtype=np.uint8))]
    wrong_magic = bytearray(blob)
    wrong_magic[0] ^= 1
    bad.append(bytes(wrong_magic))
    # a gate whose operand points forward (48-byte header: magic, version,
    # reserved, inputs, wires, gates, outputs; then the 8 W-byte wire table)
    W = int.from_bytes(blob[24:32], "little")
    fwd = bytearray(blob)
    off = 48 + 8 * W + 4  # first gate's operand a
    fwd[off:off + 4] = (W - 1).to_bytes(4, "little")
    bad.append(bytes(fwd))
    for b in bad:
        with pytest.raises(RuntimeError):
            P.Circuit.deserialize(b)


@pytest.mark.gpu
def test_key_export_import(gpu_available):
    O = oracle()
    ev, secrets, coeff, okey = oracle_setup("I_2P_LB_SR")
    P = pz()
    eng = P.Engine("I_2P_LB_SR")
    key = eng.upload_key(coeff.rgsw, coeff.autos, coeff.ksk)
    blob = key.export()
    k2 = eng.import_key(blob)
    r = O.Rng(b"\x31" * 32)
    c0 = ev.encrypt_bool(r, secrets[0], [1, 0, 1, 1])
    c1 = ev.encrypt_bool(r, secrets[0], [1, 1, 0, 1])
    gates = np.array([O.GATES[g] for g in ["nand", "xor", "or", "and"]], np.uint8)
    want = okey.gate_batch(gates, c0, c1, threads=4)
    assert np.array_equal(eng.gate_batch(key, gates, c0, c1), want)
    assert np.array_equal(eng.gate_batch(k2, gates, c0, c1), want)
    other_root = P.Engine("I_2P_LB_SR", ntt_root=ev.psi())
    if other_root.ntt_root != eng.ntt_root:
        with pytest.raises(RuntimeError):
            other_root.import_key(blob)
    with pytest.raises(RuntimeError):
        P.Engine("I_4P").import_key(blob)
    with pytest.raises(RuntimeError):
        eng.import_key(blob[:-8])
