"""Oracle integer layer pinned to the reference's known-answer tests, and the
library's own integer layer checked bit-exactly against the oracle (CPU only)."""
import numpy as np
import pytest

# radix_shape.rs:240-264 (factorize_product_invariant_holds_for_smooth_sizes)
SMOOTH = [3, 5, 6, 7, 9, 10, 11, 12, 13, 14, 15, 17, 18, 21, 22, 23, 24, 25, 28, 33, 34, 35, 42, 46, 48, 49, 50,
          56, 63, 66, 69, 70, 75, 98, 100, 120, 121, 125, 143, 147, 150, 154, 176, 192, 200, 210, 231, 240, 242,
          245, 250, 253, 264, 275, 286, 294, 300, 343, 375, 384, 392, 450, 500, 506, 528, 575, 588, 600, 616, 625,
          650, 675, 686, 700, 726, 750, 784, 864, 900, 980, 1000, 1100, 1200, 1400, 1470, 1500, 1960, 2000, 2200,
          2400, 2500, 2600, 2700, 2800, 2940, 3000, 4000, 4500, 5000, 6000, 7000, 7500, 10000]


def test_factorize_product_invariant(oracle):
    for n in SMOOTH:
        r = oracle.factorize_composite(n)
        assert r is not None and int(np.prod(r)) == n
        assert all(v in (2, 3, 5, 7, 11, 13, 17, 23) for v in r)


def test_factorize_pure_pow2_is_none(oracle):  # radix_shape.rs:266-275
    for e in range(1, 21):
        assert oracle.factorize_composite(1 << e) is None


def test_factorize_unsupported_is_none(oracle):  # radix_shape.rs:277-285
    for n in (19, 29, 31, 37, 38, 41, 43, 58, 361, 551):
        assert oracle.factorize_composite(n) is None


def test_factorize_innermost_first(oracle):  # radix_shape.rs:288-298
    assert oracle.factorize_composite(24)[0] == 3
    assert oracle.factorize_composite(28)[0] == 7
    assert oracle.factorize_composite(46)[0] == 23


def test_radix4_lowering_kat(oracle):  # radix_shape.rs:317-324
    r = oracle.factorize_composite(192)
    assert r == [3, 2, 2, 2, 2, 2, 2]
    assert oracle.lower_radix2_pairs_to_radix4(r) == [3, 4, 4, 4]
    assert oracle.lower_radix2_pairs_to_radix4([2, 2, 2]) == [4, 2]


def test_primitive_root_table_matches_search(oracle):  # rader/mod.rs:449-458
    for p in (3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53, 59, 61, 67, 71, 73, 79, 83, 89, 97, 101,
              109, 113, 127, 131, 151, 167, 173, 179, 181, 193, 197, 199, 10007):
        assert oracle.primitive_root(p) == oracle.primitive_root_dynamic(p)


def test_inverse_generator_order_identity(oracle):  # rader/mod.rs:460-476
    for p in (5, 7, 11, 13, 17, 97, 1009, 2053):
        g = oracle.primitive_root(p)
        gi = oracle.inverse_mod(g, p)
        order = oracle.generator_order(p, g)
        inv = oracle.inverse_generator_order(p, g)
        for q in range(p - 1):
            assert inv[q] == pow(gi, q, p)
            assert (order[q] * inv[q]) % p == 1


def test_twiddle_table_layout(oracle):  # twiddle_table.rs:206-261
    for n in (2, 4, 8, 64, 1024):
        t = oracle.twiddle_table(n, -1.0)
        assert len(t) == n - 1
        ti = oracle.twiddle_table(n, 1.0)
        np.testing.assert_allclose(ti, np.conj(t), atol=0)
        off = 0
        length = 2
        while length <= n:
            half = length // 2
            ref = np.exp(-2j * np.pi * np.arange(half) / length)
            np.testing.assert_allclose(t[off:off + half], ref, atol=1e-13)
            off += half
            length *= 2


def test_short_winograd_membership(oracle):  # traits.rs:351-391
    sizes = set(range(2, 57)) | {58, 60, 62, 63, 64, 81, 128}
    for n in range(1, 300):
        assert oracle.is_short_winograd(n) == (n in sizes)


def test_pfa_perms_are_bijections(oracle):  # misc.rs:233-256
    for n1, n2 in ((3, 4), (5, 2), (125, 2), (7, 9), (16, 9), (11, 13)):
        a, b = oracle.pfa_perm(n1, n2)
        n = n1 * n2
        assert sorted(a.tolist()) == list(range(n))
        assert sorted(b.tolist()) == list(range(n))


def test_dispatch_strategies_of_workload_lengths(oracle):
    assert oracle.dispatch_strategy(4096) == "four_step"
    assert oracle.four_step_split(4096) == (64, 64)
    assert oracle.dispatch_strategy(256) == "stockham"
    assert oracle.dispatch_strategy(243) == "composite"
    assert oracle.prime23_radices(243) == [3, 3, 3, 3, 3]
    assert oracle.dispatch_strategy(250) == "composite"
    assert oracle.prime23_radices(250) == [5, 5, 5, 2]
    assert oracle.coprime_factors(250) == (125, 2)
    assert oracle.dispatch_strategy(343) == "composite"
    assert oracle.prime23_radices(343) == [7, 7, 7]
    assert oracle.dispatch_strategy(1009) == "rader_full"
    assert oracle.dispatch_strategy(65521) == "rader_half"
    assert oracle.dispatch_strategy(361) == "untransformed"
    assert oracle.dispatch_strategy(30) == "winograd"


LENGTHS = list(range(1, 600)) + [1009, 1024, 2048, 2053, 4096, 4099, 10007, 16384, 30030, 65521, 65536, 1 << 20]


def test_library_integer_layer_matches_oracle(oracle, afc):
    for n in LENGTHS:
        info = afc.length_info(n)
        assert info["strategy"] == oracle.dispatch_strategy(n), n
        assert info["radices"] == oracle.prime23_radices(n), n
        assert info["coprime"] == oracle.coprime_factors(n), n
        if n > 1 and (n & (n - 1)) == 0:
            assert info["four_step"] == oracle.four_step_split(n)
        assert info["is_prime"] == oracle.is_prime(n)
        if info["is_prime"]:
            g = oracle.primitive_root(n)
            assert info["primitive_root"] == g
            assert info["primitive_root_inv"] == oracle.inverse_mod(g, n)
        assert info["is_short_winograd"] == oracle.is_short_winograd(n)
        cop = oracle.coprime_factors(n)
        assert info["has_static_coprime_codelet"] == (bool(cop) and oracle.has_static_coprime_codelet(*cop))


@pytest.mark.parametrize("p", [3, 5, 7, 11, 97, 1009, 1031, 2053, 10007, 65521])
def test_library_rader_maps_match_oracle(oracle, afc, p):
    g = oracle.primitive_root(p)
    gather, scatter = afc.rader_maps(p)
    np.testing.assert_array_equal(gather, oracle.generator_order(p, g))
    np.testing.assert_array_equal(scatter, oracle.inverse_generator_order(p, g))


@pytest.mark.parametrize("n1,n2", [(3, 4), (5, 2), (125, 2), (7, 9), (16, 9), (11, 13), (343, 8)])
def test_library_pfa_perm_matches_oracle(oracle, afc, n1, n2):
    a, b = afc.pfa_perm(n1, n2)
    oa, ob = oracle.pfa_perm(n1, n2)
    np.testing.assert_array_equal(a, oa)
    np.testing.assert_array_equal(b, ob)


# The GPU stage factorization (this library's choice, not the reference's):
# fewest stages over the register butterflies 2..16, composites 6, 9, 10, 12,
# 14, 15 nested; powers of two keep radix 16 stages then one of 8 / 4 / 2.
@pytest.mark.parametrize("n,rad", [(4096, [16, 16, 16]), (2048, [16, 16, 8]), (243, [9, 9, 3]),
                                   (250, [10, 5, 5]), (343, [7, 7, 7]), (1000, [10, 10, 10]),
                                   (45, [9, 5]), (12, [12]), (6, [6]), (2310, [11, 15, 14])])
def test_gpu_stage_radices(afc, n, rad):
    info = afc.length_info(n)
    got = info["gpu_radices"]
    assert sorted(got) == sorted(rad), (n, got)
    assert int(np.prod(got)) == n
