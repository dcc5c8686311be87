"""Request-frame helpers shared by the tests and the golden-vector script: the malformed-frame table and the
seeded mutation of tests/engine.rs (reference), restated."""
import numpy as np

Q = 4294955009
MUTATION_SEED = 0x5EEDF00D  # tests/engine.rs:170


def mix(state):
    """synthetic::mix (src/service.rs:46-52) on a one-element list holding the state."""
    state[0] = (state[0] + 0x9E3779B97F4A7C15) & 0xFFFFFFFFFFFFFFFF
    z = state[0]
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & 0xFFFFFFFFFFFFFFFF
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & 0xFFFFFFFFFFFFFFFF
    return z ^ (z >> 31)


def mutate(valid, rnd, count, q=Q):
    """mutate (tests/engine.rs:29-68): one of eight seeded corruptions of a valid frame."""
    v = bytearray(bytes(valid))
    special = [0, 1, (q - 1) & 0xFFFFFFFF, q & 0xFFFFFFFF, (q + 1) & 0xFFFFFFFF, 0xFFFFFFFF, 1 << 31]
    kind = rnd() % 8
    if kind == 0:
        del v[rnd() % len(v):]
    elif kind == 1:
        for _ in range(1 + rnd() % 64):
            v.append(rnd() & 0xFF)
    elif kind == 2:
        i = rnd() % 13
        v[i] = rnd() & 0xFF
    elif kind == 3:
        i = rnd() % 13
        v[i] ^= 1 << (rnd() % 8)
    elif kind == 4:
        w = 9 + 4 * (rnd() % (2 * count))
        x = special[rnd() % len(special)]
        v[w:w + 4] = x.to_bytes(4, "little")
    elif kind == 5:
        nq = (len(v) - 9 - 8 * count) // 4
        w = 9 + 8 * count + 4 * (rnd() % nq)
        x = special[rnd() % len(special)]
        v[w:w + 4] = x.to_bytes(4, "little")
    elif kind == 6:
        i = rnd() % len(v)
        v[i] ^= 1 << (rnd() % 8)
    return np.frombuffer(bytes(v), dtype=np.uint8).copy()


def malformed_table(r0, r1, count, q=Q):
    """The eight hand-built frames of tests/engine.rs:130-148 and their expected statuses."""
    frames = [r0.copy(), r0[:-1].copy(), np.concatenate([r0, np.zeros(1, np.uint8)])]
    v = r0.copy(); v[0] = 1; frames.append(v)
    v = r0.copy(); v[1:5] = np.frombuffer((0xFFFFFFFF).to_bytes(4, "little"), np.uint8); frames.append(v)
    v = r0.copy(); v[9:13] = np.frombuffer(q.to_bytes(4, "little"), np.uint8); frames.append(v)
    v = r0.copy(); off = 9 + 8 * count - 4; v[off:off + 4] = 0xFF; frames.append(v)
    frames.append(r1.copy())
    return frames, [0, 1, 1, 2, 2, 3, 3, 0]


def mutated_batches(base, count, batches=8, per=64):
    """8 batches of 64 seeded mutations of the base frames (tests/engine.rs:170-192)."""
    state = [MUTATION_SEED]
    rnd = lambda: mix(state)
    out = []
    for _ in range(batches):
        fr = []
        for _ in range(per):
            k = rnd() % len(base)
            fr.append(mutate(base[k], rnd, count))
        out.append(fr)
    return out
