"""stark_info_new / the prover-buffer map, on the host (no device call).

The library parses a setup's starkinfo JSON (StarkInfo::load, stark_info.cpp:24-263) and lays out the
prover buffer as StarkInfo::setMapOffsets does (stark_info.cpp:450-670) so that commit_witness can
land the stage-1 LDE at mapOffsets[("cm1", true)] and its tree at ("mt1", true), as the reference's
later stages expect.  The expected offsets below are worked out by hand from those lines for one
small setup; each step of the arithmetic is written next to its number.
"""
import json
import os
import tempfile

import pytest

# N = 2^10, NExt = 2^11, arity 4.  Tree nodes of 2048 leaves: 2048 + 512 + 128 + 32 + 8 + 2 + 2 (zero
# padding of the 2-node level) + 1 = 2733 digests = 10932 words.
SETUP = {
    "name": "Example",
    "starkStruct": {"nBits": 10, "nBitsExt": 11, "nQueries": 8, "verificationHashType": "GL", "merkleTreeArity": 4,
                    "transcriptArity": 4, "merkleTreeCustom": False, "lastLevelVerification": 1, "powBits": 0,
                    "hashCommits": True, "steps": [{"nBits": 11}, {"nBits": 7}, {"nBits": 3}]},
    "nPublics": 3, "nConstants": 5, "nStages": 2, "qDeg": 2, "qDim": 3, "nConstraints": 1, "friExpId": 0,
    "cExpId": 1, "customCommits": [], "openingPoints": [0, 1], "boundaries": [{"name": "everyRow"}],
    "challengesMap": [{"stage": 2, "name": "std_alpha", "dim": 3, "stageId": i} for i in range(4)],
    "publicsMap": [{"name": "p%d" % i} for i in range(3)],
    "airgroupValuesMap": [{"name": "gsum", "stage": 2}],
    "airValuesMap": [{"name": "a", "stage": 1}, {"name": "b", "stage": 2}],
    "proofValuesMap": [],
    "cmPolsMap": [], "customCommitsMap": [], "constPolsMap": [],
    "evMap": [{"type": "cm", "id": i, "prime": 0} for i in range(6)],
    "mapSectionsN": {"const": 5, "cm1": 7, "cm2": 4, "cm3": 6},
}

# StarkInfo::setMapOffsets with gpu = true, preallocate = false, recursive = false:
#   const tree   0, += 2048*5 + 10932                       -> 21172
#   const        21172, += 1024*5                           -> 26292
#   publics 3, airgroupvalues 3 (one stage-2 value), airvalues 1 + 3, challenge 4, nonce 1,
#   nonce_blocks (2^19 + 511) / 512 = 1024, input_hash_nonce 4, evals 6*3, challenges 4*3,
#   xdivxsub 2*3, fri_queries 8, fri_queries_perm (8*11 + 62) / 63 = 2   -> 27381
#   proof_queries: maxTreeWidth max(7, 16*3, 16*3) = 48; siblings ceil(11/2) - 1 = 5 levels of 3*4
#   words -> 108 words per tree; (1 + 3 + 0 trees + 2 FRI trees) * 108 * 8 queries = 5184 -> 32565
#   cm1 extended 32565, += 2048*7 = 14336                   -> 46901
#   mt1          46901, += 10932                            -> 57833
#   cm1          57833; contributions = 57833 + 1024*7      =  65001
#   cm2 ext 57833 (+8192), mt2 66025 (+10932) -> 76957; cm2 = cm3 ext = 76957 (+12288), mt3 89245
#   (+10932) -> 100177; q = f = 100177 (+6144) -> 106321; buff_helper 106321 (+6144) -> 112465;
#   fri_1 112465 (+128*48), mt_fri_1 118609 (+692) -> 119301; fri_2 (+8*48), mt_fri_2 119685 (+52)
#   -> 119737 = mapTotalN (the helper maxima stop at 112467)
EXPECT_PROVER = {("cm1", True): 32565, ("mt1", True): 46901, ("cm1", False): 57833, ("const", True): 0,
                 ("const", False): 21172, ("publics", False): 26292, ("proof_queries", False): 27381,
                 ("cm2", False): 76957, ("q", True): 100177, ("buff_helper", False): 106321,
                 ("fri_1", True): 112465, ("mt_fri_2", True): 119685}

# the verifier map (load, stark_info.cpp:265-282): cm stages of nQueries rows: 7*8, 4*8, 6*8
EXPECT_VERIFY = {("cm1", False): 0, ("cm2", False): 56, ("cm3", False): 88}

# the constraint checker's map with gpu (stark_info.cpp:283-341): const 1024*5 = 5120; constraints
# 5120 (+3072); publics 8192 (+3); airgroupvalues 8195 (+3); airvalues 8198 (+4); challenge 8202 (+6);
# cm1 8208 (+7168); cm2 15376 (+4096); q 19472 (+3072) -> mem_exps 22544 = mapTotalN
EXPECT_CONSTRAINTS = {("constraints", False): 5120, ("publics", False): 8192, ("cm1", False): 8208,
                      ("cm2", False): 15376, ("q", True): 19472, ("mem_exps", False): 22544}


@pytest.fixture(scope="module")
def setup_file():
    d = tempfile.mkdtemp()
    path = os.path.join(d, "example.starkinfo.json")
    with open(path, "w") as f:
        json.dump(SETUP, f, indent=1)
    return path


def test_parse_fields(pkg, setup_file):
    si = pkg.StarkInfo(setup_file)
    assert si.value("nBits") == 10 and si.value("nBitsExt") == 11
    assert si.value("merkleTreeArity") == 4 and si.value("lastLevelVerification") == 1
    assert si.value("nConstants") == 5 and si.value("qDeg") == 2 and si.value("qDim") == 3
    assert si.value("mapSectionsN.cm1") == 7 and si.value("mapSectionsN.cm3") == 6
    assert si.value("mapSectionsN.cm9") == 0


def test_prover_buffer_map(pkg, setup_file):
    si = pkg.StarkInfo(setup_file)
    for (sec, ext), off in EXPECT_PROVER.items():
        assert si.offset(sec, ext) == off, (sec, ext)
    assert si.map_total_n() == 119737
    assert si.map_total_n_contributions() == 65001
    lib = pkg.load()
    assert lib.get_map_total_n_custom_commits_fixed(si.ptr) == 0
    assert lib.get_const_tree_size(si.ptr) == 2048 * 5 + 10932
    assert lib.get_const_size(si.ptr) == 1024 * 5
    assert pkg.tree_num_elements(2048, 4) == 10932


def test_verifier_and_constraint_maps(pkg, setup_file):
    v = pkg.StarkInfo(setup_file, verify=True)
    for (sec, ext), off in EXPECT_VERIFY.items():
        assert v.offset(sec, ext) == off
    assert v.map_total_n() == 136
    c = pkg.StarkInfo(setup_file, verify_constraints=True)
    for (sec, ext), off in EXPECT_CONSTRAINTS.items():
        assert c.offset(sec, ext) == off
    assert c.map_total_n() == 22544


def test_preallocated_const_tree_moves_everything_down(pkg, setup_file):
    """With preallocate the const tree lives elsewhere: every later section moves down by its size."""
    p = pkg.StarkInfo(setup_file, preallocate=True)
    shift = 2048 * 5 + 10932
    assert p.offset("cm1", True) == EXPECT_PROVER[("cm1", True)] - shift
    assert p.offset("mt1", True) == EXPECT_PROVER[("mt1", True)] - shift


def test_custom_commits_fixed(pkg):
    s = json.loads(json.dumps(SETUP))
    s["customCommits"] = [{"name": "rom", "publicValues": [], "stageWidths": [3, 0, 0]}]
    s["mapSectionsN"]["rom0"] = 3
    d = tempfile.mkdtemp()
    path = os.path.join(d, "custom.starkinfo.json")
    with open(path, "w") as f:
        json.dump(s, f)
    si = pkg.StarkInfo(path)
    # rom0: N*3 source words, then NExt*3 extended words and the tree
    assert si.offset("rom0", False) == 0
    assert si.offset("rom0", True) == 1024 * 3
    assert pkg.load().get_map_total_n_custom_commits_fixed(si.ptr) == 1024 * 3 + 2048 * 3 + 10932


def test_from_shape_layout(pkg):
    si = pkg.StarkInfo.from_shape(12, 13, 9, 4)
    assert si.offset("cm1", True) == 0
    assert si.offset("mt1", True) == (1 << 13) * 9
    assert si.offset("cm1", False) == (1 << 13) * 9 + pkg.tree_num_elements(1 << 13, 4)
    assert si.value("mapSectionsN.cm1") == 9 and si.value("nConstants") == 9


@pytest.mark.parametrize("text,what", [("{", "string expected"), ("{\"a\": ", "value expected"), ('{"starkStruct": {"nBits": 3}}', "nBitsExt"),
                                      ("[1, 2", "expected"), ('{"a": tru}', "unexpected")])
def test_malformed_files_are_errors(pkg, text, what):
    d = tempfile.mkdtemp()
    path = os.path.join(d, "bad.json")
    with open(path, "w") as f:
        f.write(text)
    with pytest.raises(pkg.B200Error) as e:
        pkg.StarkInfo(path)
    assert what in str(e.value)


def test_missing_file_is_an_error(pkg):
    with pytest.raises(pkg.B200Error) as e:
        pkg.StarkInfo("/nonexistent/x.starkinfo.json")
    assert "cannot open" in str(e.value)


def test_foreign_pointers_are_refused(pkg):
    """Sizes of something that is not a StarkInfo of this library read as 0, not as garbage."""
    import ctypes
    junk = (ctypes.c_uint64 * 16)()
    lib = pkg.load()
    assert lib.get_const_tree_size(ctypes.addressof(junk)) == 0
    assert lib.get_map_total_n(ctypes.addressof(junk)) == 0
