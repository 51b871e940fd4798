"""JSON job specs (csrc/jobs.cpp) checked without a GPU: mdpd_jobs_validate, and mdpd_run_jobs
and `lmp_mdpd -jobs` on files that are refused before any device work."""
import json
import os
import subprocess

import pytest

import mdpd

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "usermeso-2.0-mdpd_b200", "lmp_mdpd")

SPEC = {
    "version": 1,
    "budget_gb": 20,
    "defaults": {"A": -40, "B": 25, "cut_r": 0.75, "dt": 0.01},
    "jobs": [
        {"name": "small", "n": 3000, "box": 8.0, "steps": 100, "seed": 3, "init_seed": 5},
        {"name": "slab", "n": 6000, "box": [16, 8, 8], "fill_hi": [8, 8, 8], "steps": 50, "exact_rng": True},
        {"name": "dpd", "style": "dpd", "n": 4000, "box": [10, 10, 10], "A": 25, "sigma": 3.0, "steps": 80},
    ],
}


def write(tmp_path, doc, name="jobs.json"):
    p = tmp_path / name
    p.write_text(doc if isinstance(doc, str) else json.dumps(doc))
    return p


def test_validate_counts_jobs_and_footprint(tmp_path):
    n, b = mdpd.validate_jobs(write(tmp_path, SPEC))
    assert n == 3
    # the same boxes through the Python spec builder: the same admission footprints
    want = (mdpd.box_bytes(mdpd.box_spec(3000, 8.0)) + mdpd.box_bytes(mdpd.box_spec(6000, (16, 8, 8), exact_rng=1)) +
            mdpd.box_bytes(mdpd.box_spec(4000, 10.0, style=1, A=25)))
    assert b == want


@pytest.mark.parametrize("edit,words", [
    (lambda d: d["jobs"][0].update(bogus=1), 'job 0 (small): unknown key "bogus"'),
    (lambda d: d.update(jobz=[]), 'top level: unknown key "jobz"'),
    (lambda d: d["jobs"][1].pop("steps"), 'job 1 (slab): "steps" is required'),
    (lambda d: d["jobs"][2].pop("box"), 'job 2 (dpd): "box" is required'),
    (lambda d: d["jobs"][0].update(n="big"), '"n" must be a number'),
    (lambda d: d["jobs"][0].update(n=1.5), '"n" must be an integer'),
    (lambda d: d["jobs"][0].update(box=[8, -1, 8]), "edges must be positive"),
    (lambda d: d["jobs"][0].update(box=[8, 8]), '"box" must be a number or a list of 3 numbers'),
    (lambda d: d["jobs"][1].update(name="small"), 'duplicate name "small"'),
    (lambda d: d["jobs"][2].update(style="sph"), '"style" must be "mdpd" or "dpd"'),
    (lambda d: d["defaults"].update(name="x"), '"name" is per job'),
    (lambda d: d["defaults"].update(gama=4.5), 'defaults: unknown key "gama"'),
    (lambda d: d.update(budget_gb=0.01), "above budget_gb"),
    (lambda d: d.update(jobs=[]), '"jobs" must list at least one job'),
    (lambda d: d["jobs"][0].update(cut=0.7), "job 0 (small): PARSE: cutA should be larger than cutB"),
])
def test_bad_specs_name_the_job_and_key(tmp_path, edit, words):
    doc = json.loads(json.dumps(SPEC))
    edit(doc)
    p = write(tmp_path, doc)
    with pytest.raises(mdpd.MdpdError) as e:
        mdpd.validate_jobs(p)
    assert e.value.code == mdpd.ERR_PARSE and words in str(e.value), str(e.value)
    # the runner refuses the same file before it touches a device, and writes nothing
    out = tmp_path / "out.jsonl"
    with pytest.raises(mdpd.MdpdError) as e2:
        mdpd.run_jobs(p, out)
    assert e2.value.code == mdpd.ERR_PARSE and words in str(e2.value)
    assert not out.exists()


def test_malformed_and_missing_files(tmp_path):
    with pytest.raises(mdpd.MdpdError) as e:
        mdpd.validate_jobs(write(tmp_path, '{"jobs": [ {"n": 10,, }]}'))
    assert e.value.code == mdpd.ERR_PARSE and "offset" in str(e.value)
    with pytest.raises(mdpd.MdpdError) as e:
        mdpd.validate_jobs(tmp_path / "none.json")
    assert e.value.code == mdpd.ERR_ARG


def test_cli_jobs_flag_reports_parse_errors(tmp_path):
    doc = json.loads(json.dumps(SPEC))
    doc["jobs"][0]["bogus"] = 1
    p = write(tmp_path, doc)
    r = subprocess.run([EXE, "-jobs", str(p), "-out", str(tmp_path / "o.jsonl")], capture_output=True, text=True)
    assert r.returncode == mdpd.ERR_PARSE and 'unknown key "bogus"' in r.stderr
