"""The cached oracle answers on the full-size workloads
(tests/golden/configs.json.gz): complete, consistent with what the workload
definitions imply, and reproducible where that is cheap on the CPU."""
import golden_configs as G

M61 = (1 << 61) - 1


def test_all_entries_present():
    d = G.load()
    for k in ("rank_uniform_16384", "rank_dependent_16384", "rank_planted_16384", "lc_planted_200000",
              "lc_iid_200000", "rank_batch_4096", "lc_batch_65536"):
        assert k in d, k


def test_entries_consistent_with_their_workloads():
    d = G.load()
    assert d["rank_uniform_16384"]["rank"] == 16384 and d["rank_uniform_16384"]["pcols_is_prefix"]
    e = d["rank_dependent_16384"]
    assert e["rank"] == 16384 - e["dep_rows"] and e["pcols_are_first_free_columns"] and len(e["dep_cols"]) == 96
    assert d["rank_planted_16384"]["rank"] == 4096
    assert d["lc_planted_200000"]["lc"] == 65280
    assert abs(d["lc_iid_200000"]["lc"] - 100000) <= 2
    import bench
    jobs, _ = bench.bm_batch_jobs()
    lcs = d["lc_batch_65536"]["lcs"]
    assert len(lcs) == len(jobs)
    assert all(lcs[i] == j[3] for i, j in enumerate(jobs) if j[2])  # planted: the order
    rjobs, _ = bench.rank_batch_jobs()
    ranks = d["rank_batch_4096"]["ranks"]
    assert len(ranks) == len(rjobs) and all(r <= j[1] for r, j in zip(ranks, rjobs))
    generic = sum(ranks[i] == (j[3] if j[2] else j[1]) for i, j in enumerate(rjobs))
    assert generic >= 0.95 * len(rjobs)


def test_long_iid_input_reproduces(O):
    e = G.entry("lc_iid_200000")
    assert G.host_sha256(O.gen_uniform(M61, e["seed"], e["n"])) == e["input_sha256"]
