"""The serving arena's best-fit allocator (host bookkeeping over one buffer; a CPU
buffer stands in for the device one)."""
import random

from cuszp_b200.serve import Arena


def test_best_fit_merges_free_blocks():
    a = Arena(4096, "cpu")
    x, y, z = a.alloc(1000), a.alloc(1000), a.alloc(1000)
    assert (x, y, z) == (0, 1024, 2048) and a.alloc(2048) == -1
    a.free(y, 1000)
    a.free(x, 1000)
    assert a.alloc(2048) == 0               # the two freed neighbours merged
    a.free(0, 2048)
    a.free(z, 1000)
    assert a.used == 0 and a.starts == [0] and a.lens == [4096] and a.by_size == [(4096, 0)]


def test_best_fit_takes_the_smallest_hole():
    a = Arena(8192, "cpu")
    blocks = [a.alloc(1024) for _ in range(8)]
    a.free(blocks[1], 1024)                 # holes of 1, 2 and 3 blocks
    a.free(blocks[3], 2048)
    a.free(blocks[6], 1024)
    a.free(blocks[7], 1024)
    assert a.alloc(1500) == blocks[3]       # the 2-block hole, not the first or the last
    assert a.alloc(2048) == blocks[6]


def test_random_alloc_free_against_a_model():
    """Allocations never overlap each other or leave the buffer, a failed allocation
    means no free block is large enough, free blocks stay disjoint and merged, and the
    size index always lists exactly the free blocks; frees include the tail-only frees
    compress results make."""
    rng = random.Random(1)
    for _ in range(60):
        a = Arena(1 << 20, "cpu")
        live = {}
        for _ in range(300):
            if live and rng.random() < 0.45:
                off = rng.choice(list(live))
                n = live.pop(off)
                r = Arena.rounded(n)
                if r > 512 and rng.random() < 0.5:
                    keep = Arena.rounded(rng.randint(1, r - 256))
                    if keep < r:
                        a.free(off + keep, r - keep)
                        live[off] = keep
                        continue
                a.free(off, n)
            else:
                n = rng.randint(1, 40000)
                off = a.alloc(n)
                if off < 0:
                    assert max(a.lens, default=0) < Arena.rounded(n)
                else:
                    end = off + Arena.rounded(n)
                    assert end <= a.size
                    for o, m in live.items():
                        assert end <= o or o + Arena.rounded(m) <= off
                    live[off] = n
            assert sorted(zip(a.lens, a.starts)) == a.by_size
            for i in range(len(a.starts) - 1):
                assert a.starts[i] + a.lens[i] < a.starts[i + 1]
            assert a.used + sum(a.lens) == a.size
