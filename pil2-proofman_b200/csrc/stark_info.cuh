// The StarkInfo the commit entry points read, and the prover-buffer map they write into.
//
// proofman hands commit_witness a `SetupC {p_stark_info, p_expressions_bin}` (common/src/setup.rs:45-57),
// read by the reference as `SetupCtx {StarkInfo &, ExpressionsBin &}` (setup_ctx.hpp:200-207), where
// p_stark_info comes from stark_info_new(filename, ...) (starks_api.hpp:37).  This file is that
// object for this library: stark_info_new parses the setup's starkinfo JSON for the fields the
// commit and the buffer map depend on (StarkInfo::load, stark_info.cpp:24-263) and lays out the
// prover buffer as StarkInfo::setMapOffsets does (stark_info.cpp:450-670; the verifier and
// constraint-check variants of load, :265-340), so the stage-1 LDE lands at
// mapOffsets[("cm1", true)], its tree at mapOffsets[("mt1", true)] and the column-major trace at
// mapOffsets[("cm1", false)] of a stream's buffer, where the reference's later stages look for them.
// Host code only.
#pragma once
#include <cmath>
#include <cstdint>
#include <fstream>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <thread>
#include <utility>
#include <vector>

namespace sinfo {

// ------------------------------------------------------------------ JSON ----
// A small recursive-descent reader: objects, arrays, strings (escapes kept literal except \" and
// \\), numbers (integers exactly, others as double), true/false/null.  Enough for starkinfo files.
struct Json {
    enum Kind { NUL, BOOL, NUM, STR, ARR, OBJ } kind = NUL;
    bool b = false;
    bool is_int = false;
    int64_t i = 0;
    double d = 0;
    std::string s;
    std::vector<Json> a;
    std::vector<std::pair<std::string, Json>> o;

    const Json *get(const std::string &k) const
    {
        if (kind != OBJ) return nullptr;
        for (const auto &kv : o)
            if (kv.first == k) return &kv.second;
        return nullptr;
    }
    size_t size() const { return kind == ARR ? a.size() : kind == OBJ ? o.size() : 0; }
    int64_t as_int(int64_t dflt = 0) const
    {
        if (kind == NUM) return is_int ? i : (int64_t)d;
        if (kind == BOOL) return b ? 1 : 0;
        return dflt;
    }
};

class JsonReader {
public:
    explicit JsonReader(const std::string &t) : t_(t) {}
    bool parse(Json &out, std::string &err)
    {
        try {
            out = value();
            ws();
            if (p_ != t_.size()) fail("trailing characters");
            return true;
        } catch (const std::string &e) {
            err = e;
            return false;
        }
    }

private:
    const std::string &t_;
    size_t p_ = 0;
    [[noreturn]] void fail(const char *what) { throw std::string(what) + " at byte " + std::to_string(p_); }
    void ws()
    {
        while (p_ < t_.size() && (t_[p_] == ' ' || t_[p_] == '\n' || t_[p_] == '\r' || t_[p_] == '\t')) p_++;
    }
    bool lit(const char *w)
    {
        size_t n = std::char_traits<char>::length(w);
        if (t_.compare(p_, n, w) != 0) return false;
        p_ += n;
        return true;
    }
    std::string str()
    {
        if (t_[p_] != '"') fail("string expected");
        std::string s;
        for (p_++; p_ < t_.size() && t_[p_] != '"'; p_++) {
            if (t_[p_] == '\\' && p_ + 1 < t_.size()) {
                p_++;
                if (t_[p_] != '"' && t_[p_] != '\\') s.push_back('\\');
            }
            s.push_back(t_[p_]);
        }
        if (p_ >= t_.size()) fail("unterminated string");
        p_++;
        return s;
    }
    Json value()
    {
        ws();
        if (p_ >= t_.size()) fail("value expected");
        Json v;
        const char c = t_[p_];
        if (c == '{') {
            v.kind = Json::OBJ;
            p_++;
            ws();
            if (t_[p_] == '}') {
                p_++;
                return v;
            }
            for (;;) {
                ws();
                std::string k = str();
                ws();
                if (t_[p_] != ':') fail("':' expected");
                p_++;
                v.o.emplace_back(std::move(k), value());
                ws();
                if (t_[p_] == ',') {
                    p_++;
                    continue;
                }
                if (t_[p_] == '}') {
                    p_++;
                    return v;
                }
                fail("',' or '}' expected");
            }
        }
        if (c == '[') {
            v.kind = Json::ARR;
            p_++;
            ws();
            if (t_[p_] == ']') {
                p_++;
                return v;
            }
            for (;;) {
                v.a.push_back(value());
                ws();
                if (t_[p_] == ',') {
                    p_++;
                    continue;
                }
                if (t_[p_] == ']') {
                    p_++;
                    return v;
                }
                fail("',' or ']' expected");
            }
        }
        if (c == '"') {
            v.kind = Json::STR;
            v.s = str();
            return v;
        }
        if (lit("true")) {
            v.kind = Json::BOOL;
            v.b = true;
            return v;
        }
        if (lit("false")) {
            v.kind = Json::BOOL;
            return v;
        }
        if (lit("null")) return v;
        const size_t s0 = p_;
        bool frac = false;
        if (t_[p_] == '-' || t_[p_] == '+') p_++;
        while (p_ < t_.size() && (isdigit((unsigned char)t_[p_]) || t_[p_] == '.' || t_[p_] == 'e' || t_[p_] == 'E' ||
                                  t_[p_] == '-' || t_[p_] == '+')) {
            if (!isdigit((unsigned char)t_[p_])) frac = true;
            p_++;
        }
        if (p_ == s0) fail("unexpected character");
        const std::string num = t_.substr(s0, p_ - s0);
        v.kind = Json::NUM;
        v.d = std::stod(num);
        if (!frac || (num.find_first_of(".eE") == std::string::npos)) {
            v.is_int = true;
            v.i = std::stoll(num);
        }
        return v;
    }
};

// ------------------------------------------------------------- StarkInfo ----
constexpr uint32_t MAGIC = 0x53494e46u;  // tags objects made here, so foreign pointers are refused
constexpr uint64_t HASH_SIZE = 4, FIELD_EXTENSION = 3;
constexpr uint64_t NONCES_LAUNCH_GRID_SIZE = ((1ull << 19) + 512 - 1) / 512;  // poseidon2_goldilocks.hpp:17-21

struct StarkInfo {
    uint32_t magic = MAGIC;
    // starkStruct
    uint64_t nBits = 0, nBitsExt = 0, nQueries = 0, merkleTreeArity = 4, transcriptArity = 4, lastLevelVerification = 0;
    bool merkleTreeCustom = false;
    std::string verificationHashType = "GL";
    std::vector<uint64_t> stepsBits;
    // counts and sizes
    uint64_t nPublics = 0, nConstants = 0, nStages = 2, qDeg = 0, qDim = 0;
    std::vector<std::pair<std::string, std::vector<uint64_t>>> customCommits;  // name, stageWidths
    uint64_t nOpeningPoints = 0, nBoundaries = 0, nChallenges = 0, nEvMap = 0;
    uint64_t airgroupValuesSize = 0, airValuesSize = 0, proofValuesSize = 0;
    std::map<std::string, uint64_t> mapSectionsN;
    // flags of stark_info_new
    bool recursive = false, verify_constraints = false, verify = false, gpu = true, preallocate = false,
         singleUse = false;
    // the buffer map
    std::map<std::pair<std::string, bool>, uint64_t> mapOffsets;
    uint64_t mapTotalN = 0, mapTotalNCustomCommitsFixed = 0, mapTotalNContributions = 0;
    bool calculateFixedExtended = false, constPolsAliasTree = false;

    uint64_t sectionN(const std::string &k) const
    {
        auto it = mapSectionsN.find(k);
        return it == mapSectionsN.end() ? 0 : it->second;
    }
    uint64_t offset(const std::string &k, bool ext) const
    {
        auto it = mapOffsets.find({k, ext});
        return it == mapOffsets.end() ? UINT64_MAX : it->second;
    }
    // MerkleTreeGL::getNumNodes / StarkInfo::getNumNodesMT (stark_info.cpp:736-749)
    uint64_t numNodesMT(uint64_t height) const
    {
        uint64_t n = height, level = height;
        const uint64_t ar = merkleTreeArity;
        while (level > 1) {
            n += (ar - level % ar) % ar;
            level = (level + ar - 1) / ar;
            n += level;
        }
        return n * HASH_SIZE;
    }
    uint64_t maxTreeWidth() const
    {
        uint64_t m = 0;
        for (const auto &kv : mapSectionsN) m = std::max(m, kv.second);
        for (size_t i = 0; i + 1 < stepsBits.size(); i++) {
            const uint64_t nGroups = 1ull << stepsBits[i + 1];
            const uint64_t groupSize = (1ull << stepsBits[i]) / nGroups;
            m = std::max(m, groupSize * FIELD_EXTENSION);
        }
        return m;
    }
};

// StarkInfo::load (stark_info.cpp:24-263): the fields this file uses.  Returns "" or an error.
inline std::string load(StarkInfo &si, const Json &j)
{
    const Json *ss = j.get("starkStruct");
    if (!ss) return "starkStruct missing";
    auto num = [](const Json *o, const char *k, bool &ok) -> uint64_t {
        const Json *v = o ? o->get(k) : nullptr;
        if (!v || v->kind != Json::NUM) {
            ok = false;
            return 0;
        }
        return (uint64_t)v->as_int();
    };
    bool ok = true;
    si.nBits = num(ss, "nBits", ok);
    si.nBitsExt = num(ss, "nBitsExt", ok);
    if (!ok) return "starkStruct.nBits / nBitsExt missing";
    bool q_ok = true;
    si.nQueries = num(ss, "nQueries", q_ok);
    if (const Json *h = ss->get("verificationHashType"))
        if (h->kind == Json::STR) si.verificationHashType = h->s;
    if (si.verificationHashType == "BN128") {
        bool has = true;
        const uint64_t ar = num(ss, "merkleTreeArity", has);
        si.merkleTreeArity = has ? ar : 16;
        bool ht = true;
        const uint64_t tr = num(ss, "transcriptArity", ht);
        si.transcriptArity = has && ht ? tr : 16;
    } else {
        bool has = true;
        si.merkleTreeArity = num(ss, "merkleTreeArity", has);
        if (!has) return "starkStruct.merkleTreeArity missing";
        bool ht = true;
        si.transcriptArity = num(ss, "transcriptArity", ht);
    }
    if (const Json *v = ss->get("merkleTreeCustom")) si.merkleTreeCustom = v->as_int() != 0;
    if (const Json *v = ss->get("lastLevelVerification")) si.lastLevelVerification = (uint64_t)v->as_int();
    if (const Json *st = ss->get("steps"))
        for (const Json &s : st->a)
            if (const Json *b = s.get("nBits")) si.stepsBits.push_back((uint64_t)b->as_int());
    auto top = [&](const char *k) -> uint64_t {
        const Json *v = j.get(k);
        return v ? (uint64_t)v->as_int() : 0;
    };
    si.nPublics = top("nPublics");
    si.nConstants = top("nConstants");
    si.nStages = j.get("nStages") ? top("nStages") : 2;
    si.qDeg = top("qDeg");
    si.qDim = top("qDim");
    if (const Json *cc = j.get("customCommits"))
        for (const Json &c : cc->a) {
            std::pair<std::string, std::vector<uint64_t>> e;
            if (const Json *n = c.get("name")) e.first = n->s;
            if (const Json *w = c.get("stageWidths"))
                for (const Json &x : w->a) e.second.push_back((uint64_t)x.as_int());
            si.customCommits.push_back(e);
        }
    auto count = [&](const char *k) -> uint64_t {
        const Json *v = j.get(k);
        return v ? v->size() : 0;
    };
    si.nOpeningPoints = count("openingPoints");
    si.nBoundaries = count("boundaries");
    si.nChallenges = count("challengesMap");
    si.nEvMap = count("evMap");
    // values maps: stage 1 entries take one word, the others a cubic extension element
    auto values_size = [&](const char *k) -> uint64_t {
        uint64_t n = 0;
        if (const Json *m = j.get(k))
            for (const Json &e : m->a) {
                const Json *st = e.get("stage");
                n += (st && st->as_int() == 1) ? 1 : FIELD_EXTENSION;
            }
        return n;
    };
    si.airgroupValuesSize = values_size("airgroupValuesMap");
    si.airValuesSize = values_size("airValuesMap");
    si.proofValuesSize = values_size("proofValuesMap");
    if (const Json *m = j.get("mapSectionsN"))
        for (const auto &kv : m->o) si.mapSectionsN[kv.first] = (uint64_t)kv.second.as_int();
    if (si.sectionN("cm1") == 0 && !j.get("mapSectionsN")) return "mapSectionsN missing";
    return "";
}

// StarkInfo::setMapOffsets (stark_info.cpp:450-670), the prover-buffer map.
inline void set_map_offsets(StarkInfo &si)
{
    auto &mo = si.mapOffsets;
    const uint64_t N = 1ull << si.nBits, NExt = 1ull << si.nBitsExt;
    mo[{"const", false}] = 0;
    mo[{"const", true}] = 0;
    mo[{"cm1", false}] = 0;
    si.mapTotalNCustomCommitsFixed = 0;
    for (const auto &c : si.customCommits)
        if (!c.second.empty() && c.second[0] > 0) {
            mo[{c.first + "0", false}] = si.mapTotalNCustomCommitsFixed;
            si.mapTotalNCustomCommitsFixed += c.second[0] * N;
            mo[{c.first + "0", true}] = si.mapTotalNCustomCommitsFixed;
            si.mapTotalNCustomCommitsFixed += c.second[0] * NExt + si.numNodesMT(NExt);
        }
    uint64_t &T = si.mapTotalN;
    T = 0;
    const uint64_t numNodes = si.numNodesMT(NExt);
    if (!si.preallocate && si.gpu) {
        mo[{"const", true}] = T;
        T += NExt * si.nConstants + numNodes;
        if (!si.recursive && (NExt * si.nConstants * 8.0 / (1024 * 1024)) >= 512) si.calculateFixedExtended = true;
        si.constPolsAliasTree = si.singleUse && si.calculateFixedExtended;
    }
    if (si.gpu) {
        if (si.constPolsAliasTree) {
            mo[{"const", false}] = mo[{"const", true}];
        } else {
            mo[{"const", false}] = T;
            T += N * si.nConstants;
        }
        mo[{"custom_fixed", false}] = T;
        T += si.mapTotalNCustomCommitsFixed;
        mo[{"publics", false}] = T;
        T += si.nPublics;
        mo[{"proofvalues", false}] = T;
        T += si.proofValuesSize;
        mo[{"airgroupvalues", false}] = T;
        T += si.airgroupValuesSize;
        mo[{"airvalues", false}] = T;
        T += si.airValuesSize;
        mo[{"challenge", false}] = T;
        T += HASH_SIZE;
        mo[{"nonce", false}] = T;
        T += 1;
        mo[{"nonce_blocks", false}] = T;
        T += NONCES_LAUNCH_GRID_SIZE;
        const bool bn = si.verificationHashType == "BN128";
        if (bn) T = ((T + 3) / 4) * 4;
        mo[{"input_hash_nonce", false}] = T;
        T += bn ? 12 : HASH_SIZE;
        mo[{"evals", false}] = T;
        T += si.nEvMap * FIELD_EXTENSION;
        mo[{"challenges", false}] = T;
        T += si.nChallenges * FIELD_EXTENSION;
        mo[{"xdivxsub", false}] = T;
        T += si.nOpeningPoints * FIELD_EXTENSION;
        mo[{"fri_queries", false}] = T;
        T += si.nQueries;
        const uint64_t permBits = si.stepsBits.empty() ? 0 : si.stepsBits[0];
        mo[{"fri_queries_perm", false}] = T;
        T += (si.nQueries * permBits + 62) / 63;
        const uint64_t maxTreeWidth = si.maxTreeWidth();
        const uint64_t nSiblings =
            (uint64_t)std::ceil((double)si.nBitsExt / std::log2((double)si.merkleTreeArity)) - si.lastLevelVerification;
        const uint64_t perLevel = bn ? si.merkleTreeArity * 4 : (si.merkleTreeArity - 1) * HASH_SIZE;
        const uint64_t maxProofBuffSize = maxTreeWidth + nSiblings * perLevel;
        const uint64_t nTrees = 1 + (si.nStages + 1) + si.customCommits.size();
        const uint64_t nTreesFRI = si.stepsBits.empty() ? 0 : si.stepsBits.size() - 1;
        mo[{"proof_queries", false}] = T;
        T += (nTrees + nTreesFRI) * maxProofBuffSize * si.nQueries;
    }
    uint64_t maxTotalN = 0;
    mo[{"cm1", true}] = T;
    T += NExt * si.sectionN("cm1");
    mo[{"mt1", true}] = T;
    T += numNodes;
    mo[{"cm1", false}] = T;
    si.mapTotalNContributions = si.recursive ? 0 : T + N * si.sectionN("cm1");
    mo[{"cm2", true}] = T;
    T += NExt * si.sectionN("cm2");
    mo[{"mt2", true}] = T;
    T += numNodes;
    T = std::max(mo[{"cm1", false}] + N * si.sectionN("cm1"), T);
    mo[{"cm2", false}] = T;
    mo[{"cm3", true}] = T;
    T += NExt * si.sectionN("cm3");
    mo[{"mt3", true}] = T;
    T += numNodes;
    if (!si.gpu) {
        mo[{"evals", true}] = T;
        T += si.nEvMap * std::max(1u, std::thread::hardware_concurrency()) * FIELD_EXTENSION;
    }
    T = std::max(mo[{"cm2", false}] + N * si.sectionN("cm2"), T);
    mo[{"f", true}] = T;
    mo[{"q", true}] = T;
    T += NExt * FIELD_EXTENSION;
    mo[{"constraints", false}] = mo[{"q", true}];
    uint64_t maxSizeHelper = 0;
    if (si.gpu) {
        maxSizeHelper += si.nBoundaries * NExt;
        mo[{"zi", true}] = T;
        mo[{"x", true}] = T;
    }
    maxTotalN = std::max(maxTotalN, T + maxSizeHelper);
    mo[{"mem_exps", false}] = T + maxSizeHelper;
    uint64_t LEvSize = mo[{"f", true}];
    mo[{"lev", false}] = LEvSize;
    const uint64_t maxOpenings = std::min<uint64_t>(si.nOpeningPoints, 4);
    LEvSize += maxOpenings * N * FIELD_EXTENSION;
    if (!si.gpu) {
        mo[{"buff_helper_fft_lev", false}] = LEvSize;
        LEvSize += maxOpenings * N * FIELD_EXTENSION;
    } else {
        mo[{"extra_helper_fft_lev", false}] = LEvSize;
        LEvSize += FIELD_EXTENSION * N + si.nOpeningPoints * FIELD_EXTENSION;
    }
    maxTotalN = std::max(maxTotalN, LEvSize);
    mo[{"buff_helper", false}] = T;
    T += NExt * FIELD_EXTENSION;
    if (!si.gpu) {
        uint64_t s2 = mo[{"cm2", false}] + N * si.sectionN("cm2");
        mo[{"buff_helper_fft_2", false}] = s2;
        s2 += NExt * si.sectionN("cm2");
        maxTotalN = std::max(maxTotalN, s2);
        uint64_t s1 = mo[{"cm1", false}] + N * si.sectionN("cm1");
        mo[{"buff_helper_fft_1", false}] = s1;
        s1 += NExt * si.sectionN("cm1");
        maxTotalN = std::max(maxTotalN, s1);
        uint64_t sq = mo[{"q", true}] + NExt * FIELD_EXTENSION;
        mo[{"buff_helper_fft_" + std::to_string(si.nStages + 1), false}] = sq;
        sq += NExt * si.sectionN("cm" + std::to_string(si.nStages + 1));
        maxTotalN = std::max(maxTotalN, sq);
    } else {
        uint64_t sq = mo[{"q", true}] + NExt * FIELD_EXTENSION;
        mo[{"extra_helper_fft", false}] = sq;
        sq += NExt * FIELD_EXTENSION + si.qDeg;
        maxTotalN = std::max(maxTotalN, sq);
    }
    for (size_t step = 0; step + 1 < si.stepsBits.size(); step++) {
        const uint64_t height = 1ull << si.stepsBits[step + 1];
        const uint64_t width = ((1ull << si.stepsBits[step]) / height) * FIELD_EXTENSION;
        mo[{"fri_" + std::to_string(step + 1), true}] = T;
        T += height * width;
        if (si.verificationHashType == "GL") {
            mo[{"mt_fri_" + std::to_string(step + 1), true}] = T;
            T += si.numNodesMT(height);
        }
    }
    T = std::max(T, maxTotalN);
}

// The tail of StarkInfo::load (stark_info.cpp:265-341): the verifier's and the constraint checker's
// buffer maps, else setMapOffsets.
inline void buffer_map(StarkInfo &si)
{
    auto &mo = si.mapOffsets;
    const uint64_t N = 1ull << si.nBits, NExt = 1ull << si.nBitsExt;
    if (si.verify) {
        si.gpu = false;
        si.mapTotalN = si.mapTotalNCustomCommitsFixed = si.mapTotalNContributions = 0;
        mo[{"const", false}] = 0;
        for (uint64_t stage = 1; stage <= si.nStages + 1; ++stage) {
            mo[{"cm" + std::to_string(stage), false}] = si.mapTotalN;
            si.mapTotalN += si.sectionN("cm" + std::to_string(stage)) * si.nQueries;
        }
        for (const auto &c : si.customCommits)
            if (!c.second.empty() && c.second[0] > 0) {
                mo[{c.first + "0", false}] = si.mapTotalNCustomCommitsFixed;
                si.mapTotalNCustomCommitsFixed += c.second[0] * si.nQueries;
            }
    } else if (si.verify_constraints) {
        si.mapTotalN = 0;
        if (si.gpu) {
            mo[{"const", false}] = 0;
            si.mapTotalN += N * si.nConstants;
        }
        si.mapTotalNCustomCommitsFixed = si.mapTotalNContributions = 0;
        for (const auto &c : si.customCommits)
            if (!c.second.empty() && c.second[0] > 0) {
                mo[{c.first + "0", false}] = si.mapTotalNCustomCommitsFixed;
                si.mapTotalNCustomCommitsFixed += c.second[0] * N;
                mo[{c.first + "0", true}] = si.mapTotalNCustomCommitsFixed;
                si.mapTotalNCustomCommitsFixed += c.second[0] * NExt + si.numNodesMT(NExt);
            }
        uint64_t &T = si.mapTotalN;
        if (si.gpu) {
            mo[{"constraints", false}] = T;
            T += N * 3;
            mo[{"custom_fixed", false}] = T;
            T += si.mapTotalNCustomCommitsFixed;
            mo[{"publics", false}] = T;
            T += si.nPublics;
            mo[{"proofvalues", false}] = T;
            T += si.proofValuesSize;
            mo[{"airgroupvalues", false}] = T;
            T += si.airgroupValuesSize;
            mo[{"airvalues", false}] = T;
            T += si.airValuesSize;
            mo[{"challenge", false}] = T;
            T += 2 * FIELD_EXTENSION;
        }
        for (uint64_t stage = 1; stage <= si.nStages; stage++) {
            mo[{"cm" + std::to_string(stage), false}] = T;
            T += N * si.sectionN("cm" + std::to_string(stage));
        }
        mo[{"q", true}] = T;
        T += N * FIELD_EXTENSION;
        mo[{"mem_exps", false}] = T;
    } else {
        set_map_offsets(si);
    }
}

// A StarkInfo for callers without a starkinfo file: the commit's four numbers, the stage-1
// contribution buffer laid out as the prover's (cm1 extended, its tree, then cm1), nothing else.
inline StarkInfo *from_shape(uint64_t nBits, uint64_t nBitsExt, uint64_t nCols, uint64_t arity)
{
    auto *si = new StarkInfo();
    si->nBits = nBits;
    si->nBitsExt = nBitsExt;
    si->merkleTreeArity = arity;
    si->nConstants = nCols;
    si->mapSectionsN["cm1"] = nCols;
    const uint64_t N = 1ull << nBits, NExt = 1ull << nBitsExt;
    si->mapOffsets[{"cm1", true}] = 0;
    si->mapOffsets[{"mt1", true}] = NExt * nCols;
    si->mapOffsets[{"cm1", false}] = NExt * nCols + si->numNodesMT(NExt);
    si->mapTotalN = si->mapTotalNContributions = si->mapOffsets[{"cm1", false}] + N * nCols;
    return si;
}

inline StarkInfo *from_file(const char *filename, std::string &err)
{
    std::ifstream f(filename ? filename : "", std::ios::binary);
    if (!f) {
        err = std::string("cannot open starkinfo file ") + (filename ? filename : "(null)");
        return nullptr;
    }
    std::stringstream ss;
    ss << f.rdbuf();
    const std::string text = ss.str();
    Json j;
    JsonReader r(text);
    if (!r.parse(j, err)) {
        err = std::string("starkinfo JSON: ") + err;
        return nullptr;
    }
    std::unique_ptr<StarkInfo> si(new StarkInfo());
    err = load(*si, j);
    if (!err.empty()) {
        err = std::string("starkinfo: ") + err;
        return nullptr;
    }
    return si.release();
}

inline StarkInfo *checked(void *p)
{
    auto *si = (StarkInfo *)p;
    return (si && si->magic == MAGIC) ? si : nullptr;
}

}  // namespace sinfo
