// SimParams3D defaults, derived constants and JSON reader.
//
// Follows simulation/parameters_sim_3d.cpp of the reference: Reset (:5-62),
// ComputeHelperVariables (:65-86), ParseFile (:89-162), ComputeLame and
// ComputeCamClayParams (:164-175). The reference parses with rapidjson; this
// file carries a small recursive-descent JSON reader of its own (objects,
// arrays, numbers, strings, literals) since only the top-level keys matter.

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/icempm_b200.h"

namespace {

// ---------------------------------------------------------------- JSON value
struct JValue {
    enum Kind { Null, Bool, Number, String, Array, Object } kind = Null;
    bool b = false;
    double num = 0;
    bool is_integer = false;   // the literal had no fraction/exponent
    std::string str;
    std::vector<JValue> arr;
    std::map<std::string, JValue> obj;
};

class JsonReader {
public:
    explicit JsonReader(const std::string& text) : s_(text), i_(0) {}

    bool parse(JValue& out) {
        skip_ws();
        if (!value(out)) return false;
        skip_ws();
        return i_ == s_.size();
    }

private:
    const std::string& s_;
    size_t i_;

    void skip_ws() {
        while (i_ < s_.size() && (s_[i_] == ' ' || s_[i_] == '\t' || s_[i_] == '\n' || s_[i_] == '\r')) ++i_;
    }
    bool literal(const char* word) {
        size_t n = std::strlen(word);
        if (s_.compare(i_, n, word) != 0) return false;
        i_ += n;
        return true;
    }
    bool value(JValue& v) {
        if (i_ >= s_.size()) return false;
        char c = s_[i_];
        if (c == '{') return object(v);
        if (c == '[') return array(v);
        if (c == '"') { v.kind = JValue::String; return string(v.str); }
        if (c == 't') { v.kind = JValue::Bool; v.b = true;  return literal("true"); }
        if (c == 'f') { v.kind = JValue::Bool; v.b = false; return literal("false"); }
        if (c == 'n') { v.kind = JValue::Null; return literal("null"); }
        return number(v);
    }
    bool number(JValue& v) {
        size_t start = i_;
        bool integer = true;
        if (i_ < s_.size() && (s_[i_] == '-' || s_[i_] == '+')) ++i_;
        bool digits = false;
        while (i_ < s_.size()) {
            char c = s_[i_];
            if (c >= '0' && c <= '9') { digits = true; ++i_; }
            else if (c == '.' || c == 'e' || c == 'E') { integer = false; ++i_; }
            else if ((c == '-' || c == '+') && (s_[i_ - 1] == 'e' || s_[i_ - 1] == 'E')) ++i_;
            else break;
        }
        if (!digits) return false;
        std::string tok = s_.substr(start, i_ - start);
        char* end = nullptr;
        v.num = std::strtod(tok.c_str(), &end);
        if (end == nullptr || *end != '\0') return false;
        v.kind = JValue::Number;
        v.is_integer = integer;
        return true;
    }
    bool string(std::string& out) {
        if (s_[i_] != '"') return false;
        ++i_;
        out.clear();
        while (i_ < s_.size() && s_[i_] != '"') {
            char c = s_[i_++];
            if (c == '\\') {
                if (i_ >= s_.size()) return false;
                char e = s_[i_++];
                switch (e) {
                    case 'n': out += '\n'; break;
                    case 't': out += '\t'; break;
                    case 'r': out += '\r'; break;
                    case 'b': out += '\b'; break;
                    case 'f': out += '\f'; break;
                    case 'u': {   // keep ASCII code points, drop the rest
                        if (i_ + 4 > s_.size()) return false;
                        unsigned cp = std::strtoul(s_.substr(i_, 4).c_str(), nullptr, 16);
                        if (cp < 128) out += (char)cp;
                        i_ += 4;
                        break;
                    }
                    default: out += e; break;
                }
            } else {
                out += c;
            }
        }
        if (i_ >= s_.size()) return false;
        ++i_;   // closing quote
        return true;
    }
    bool array(JValue& v) {
        v.kind = JValue::Array;
        ++i_;
        skip_ws();
        if (i_ < s_.size() && s_[i_] == ']') { ++i_; return true; }
        while (true) {
            JValue e;
            skip_ws();
            if (!value(e)) return false;
            v.arr.push_back(std::move(e));
            skip_ws();
            if (i_ >= s_.size()) return false;
            if (s_[i_] == ',') { ++i_; continue; }
            if (s_[i_] == ']') { ++i_; return true; }
            return false;
        }
    }
    bool object(JValue& v) {
        v.kind = JValue::Object;
        ++i_;
        skip_ws();
        if (i_ < s_.size() && s_[i_] == '}') { ++i_; return true; }
        while (true) {
            skip_ws();
            std::string key;
            if (i_ >= s_.size() || !string(key)) return false;
            skip_ws();
            if (i_ >= s_.size() || s_[i_] != ':') return false;
            ++i_;
            skip_ws();
            JValue e;
            if (!value(e)) return false;
            v.obj[key] = std::move(e);
            skip_ws();
            if (i_ >= s_.size()) return false;
            if (s_[i_] == ',') { ++i_; continue; }
            if (s_[i_] == '}') { ++i_; return true; }
            return false;
        }
    }
};

// Typed getters: rapidjson's GetInt/GetDouble on a value of the wrong type is
// an error in the reference; here it is reported as MPM_ERR_CONFIG_JSON.
bool get_int(const JValue& o, const char* key, int& out, bool& bad) {
    auto it = o.obj.find(key);
    if (it == o.obj.end()) return false;
    if (it->second.kind != JValue::Number || !it->second.is_integer) { bad = true; return false; }
    out = (int)it->second.num;
    return true;
}
bool get_double(const JValue& o, const char* key, double& out, bool& bad) {
    auto it = o.obj.find(key);
    if (it == o.obj.end()) return false;
    if (it->second.kind != JValue::Number) { bad = true; return false; }
    out = it->second.num;
    return true;
}

int parse_json_into(SimParams3D* p, const std::string& text, char* raw, int buflen) {
    mpm_params_reset(p);
    JValue doc;
    JsonReader reader(text);
    if (!reader.parse(doc) || doc.kind != JValue::Object) return MPM_ERR_CONFIG_JSON;

    bool bad = false;
    get_int(doc, "SetupType", p->SetupType, bad);

    auto rp = doc.obj.find("InputRawPoints");
    if (rp == doc.obj.end()) return MPM_ERR_CONFIG_KEY;
    if (rp->second.kind != JValue::String) return MPM_ERR_CONFIG_JSON;
    if (raw != nullptr && buflen > 0) {
        std::snprintf(raw, (size_t)buflen, "%s", rp->second.str.c_str());
    }

    auto bc = doc.obj.find("BlockCutout");
    if (bc != doc.obj.end()) {
        if (bc->second.kind != JValue::Array || bc->second.arr.size() < 3) return MPM_ERR_CONFIG_JSON;
        for (int i = 0; i < 3; i++) {
            if (bc->second.arr[i].kind != JValue::Number) return MPM_ERR_CONFIG_JSON;
            p->BlockCutout[i] = bc->second.arr[i].num;
        }
    }

    get_double(doc, "InitialTimeStep", p->InitialTimeStep, bad);
    get_double(doc, "YoungsModulus", p->YoungsModulus, bad);
    get_int(doc, "GridX", p->GridXTotal, bad);
    get_int(doc, "GridY", p->GridY, bad);
    get_int(doc, "GridZ", p->GridZ, bad);
    get_double(doc, "DomainDimensionX", p->DomainDimensionX, bad);
    get_double(doc, "ParticleViewSize", p->ParticleViewSize, bad);
    get_double(doc, "SimulationEndTime", p->SimulationEndTime, bad);
    get_double(doc, "PoissonsRatio", p->PoissonsRatio, bad);
    get_double(doc, "Gravity", p->Gravity, bad);
    get_double(doc, "Density", p->Density, bad);
    get_double(doc, "IndDiameter", p->IndDiameter, bad);
    get_double(doc, "IndVelocity", p->IndVelocity, bad);
    get_double(doc, "IndDepth", p->IndDepth, bad);

    get_double(doc, "IceCompressiveStrength", p->IceCompressiveStrength, bad);
    get_double(doc, "IceTensileStrength", p->IceTensileStrength, bad);
    get_double(doc, "IceTensileStrength2", p->IceTensileStrength2, bad);
    get_double(doc, "IceShearStrength", p->IceShearStrength, bad);

    double phi;
    if (get_double(doc, "DP_phi", phi, bad)) mpm_params_set_phi(p, phi);
    get_double(doc, "DP_threshold_p", p->DP_threshold_p, bad);
    get_double(doc, "GrainVariability", p->GrainVariability, bad);

    get_int(doc, "tpb_P2G", p->tpb_P2G, bad);
    get_int(doc, "tpb_Upd", p->tpb_Upd, bad);
    get_int(doc, "tpb_G2P", p->tpb_G2P, bad);
    get_int(doc, "GridHaloSize", p->GridHaloSize, bad);
    get_int(doc, "nPartitions", p->nPartitions, bad);

    get_double(doc, "ExtraSpaceForIncomingPoints", p->ExtraSpaceForIncomingPoints, bad);
    get_double(doc, "RebalanceThresholdFreeSpaceRemaining", p->RebalanceThresholdFreeSpaceRemaining, bad);
    get_double(doc, "RebalanceThresholdDisabledPercentage", p->RebalanceThresholdDisabledPercentage, bad);
    get_double(doc, "PointsTransferBufferFraction", p->PointsTransferBufferFraction, bad);
    get_double(doc, "animation_threshold_pos", p->animation_threshold_pos, bad);
    if (bad) return MPM_ERR_CONFIG_JSON;

    mpm_params_compute_camclay(p);
    mpm_params_compute_helper_variables(p);
    return MPM_OK;
}

}  // namespace

extern "C" {

void mpm_params_compute_lame(SimParams3D* p) {
    p->lambda = p->YoungsModulus * p->PoissonsRatio / ((1 + p->PoissonsRatio) * (1 - 2 * p->PoissonsRatio));
    p->mu = p->YoungsModulus / (2 * (1 + p->PoissonsRatio));
    p->kappa = p->mu * 2. / 3. + p->lambda;
}

void mpm_params_compute_camclay(SimParams3D* p) {
    mpm_params_compute_lame(p);
    p->NACC_beta = p->IceTensileStrength / p->IceCompressiveStrength;
}

void mpm_params_set_phi(SimParams3D* p, double phi) {
    p->DP_tan_phi = std::tan(phi * MPM_PI / 180.);
}

void mpm_params_compute_helper_variables(SimParams3D* p) {
    p->ParticleMass = p->ParticleVolume * p->Density;
    p->LiquidParticleMass = p->ParticleVolume * p->WaterDensity;
    // The reference evaluates 1.f/(200*dt) as float / double -> double.
    p->UpdateEveryNthStep = (int)(1.f / (200 * p->InitialTimeStep));
    p->cellsize = p->DomainDimensionX / p->GridXTotal;
    p->cellsize_inv = 1. / p->cellsize;
    p->Dp_inv = 4. / (p->cellsize * p->cellsize);
    p->IndRSq = p->IndDiameter * p->IndDiameter / 4.;
    p->dt_vol_Dpinv = p->InitialTimeStep * p->ParticleVolume * p->Dp_inv;
    p->dt_Gravity = p->InitialTimeStep * p->Gravity;
    p->vmax = 0.5 * p->cellsize / p->InitialTimeStep;
    p->vmax_squared = p->vmax * p->vmax;
    p->VectorCapacity_transfer = (int)(p->nPtsTotal / p->nPartitions * p->PointsTransferBufferFraction);
    p->gbOffset = p->GridZ * p->GridY * p->GridHaloSize;
    p->IndenterSubdivisions = (int)(MPM_PI * p->IndDiameter / p->cellsize);
}

void mpm_params_reset(SimParams3D* p) {
    std::memset(p, 0, sizeof(SimParams3D));
    p->nPtsTotal = 0;
    p->SimulationEndTime = 12;
    p->SimulationStep = 0;
    p->SimulationTime = 0;
    p->InitialTimeStep = 3.e-5;
    p->YoungsModulus = 5.e8;
    p->GridXTotal = 128;
    p->GridY = 55;
    p->GridZ = 55;
    p->ParticleViewSize = 2.5f;
    p->DomainDimensionX = 3.33;
    p->PoissonsRatio = 0.3;
    p->Gravity = 9.81;
    p->Density = 916;
    p->WaterDensity = 1000;
    p->DragGlobal = 0;
    p->IndDiameter = 0.324;
    p->IndVelocity = 0.2;
    p->IndDepth = 0.25;
    p->IceCompressiveStrength = 100e6;
    p->IceTensileStrength = 10e6;
    p->IceShearStrength = 6e6;
    p->IceTensileStrength2 = 5e6;
    mpm_params_set_phi(p, 45);
    p->DP_threshold_p = 1e2;
    p->tpb_P2G = 256;
    p->tpb_Upd = 512;
    p->tpb_G2P = 128;
    p->indenter_x = p->indenter_x_initial = p->indenter_y = p->indenter_y_initial = 0;
    p->SetupType = 0;
    p->GrainVariability = 0.50;
    p->GridHaloSize = 15;
    p->ExtraSpaceForIncomingPoints = 0.2;
    p->PointsTransferBufferFraction = 0.05;
    p->nPartitions = 4;
    p->RebalanceThresholdFreeSpaceRemaining = 0.10;
    p->RebalanceThresholdDisabledPercentage = 0.05;
    p->PointTransferFrequency = 2;
    p->SnapshotPeriod = 100;
    p->animation_threshold_pos = 1e-3;
    mpm_params_compute_lame(p);
    mpm_params_compute_camclay(p);
    mpm_params_compute_helper_variables(p);
}

int mpm_params_parse_string(SimParams3D* p, const char* json_text, char* raw, int buflen) {
    if (p == nullptr || json_text == nullptr) return MPM_ERR_ARG;
    return parse_json_into(p, std::string(json_text), raw, buflen);
}

int mpm_params_parse_file(SimParams3D* p, const char* path, char* raw, int buflen) {
    if (p == nullptr || path == nullptr) return MPM_ERR_ARG;
    mpm_params_reset(p);
    std::ifstream f(path, std::ios::binary);
    if (!f.good()) return MPM_ERR_CONFIG_FILE;
    std::stringstream ss;
    ss << f.rdbuf();
    return parse_json_into(p, ss.str(), raw, buflen);
}

}  // extern "C"
