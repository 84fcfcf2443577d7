// OpenFOAM ASCII case reader/writer for the DUGKS host side (see
// foam_case.hpp).  Only the subset a dugksFoam case uses is understood:
// dictionaries, counted lists, "N{value}" lists, dimension sets and the
// uniform/nonuniform field values.
#include "foam_case.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <map>
#include <sstream>
#include <sys/stat.h>

#include "dugks.h"

namespace dugks_host {

namespace {

std::string slurp(const std::string& path) {
    std::ifstream f(path, std::ios::binary);
    if (!f) throw FoamError("cannot open " + path);
    std::ostringstream ss;
    ss << f.rdbuf();
    return ss.str();
}

// comments removed, then tokens: quoted strings, single punctuation
// characters ( ) { } [ ] ; and runs of anything else
std::vector<std::string> tokenize(const std::string& text) {
    std::vector<std::string> out;
    const size_t n = text.size();
    size_t i = 0;
    while (i < n) {
        const char ch = text[i];
        if (ch == '/' && i + 1 < n && text[i + 1] == '/') {
            while (i < n && text[i] != '\n') ++i;
        } else if (ch == '/' && i + 1 < n && text[i + 1] == '*') {
            i += 2;
            while (i + 1 < n && !(text[i] == '*' && text[i + 1] == '/')) ++i;
            i += 2;
        } else if (ch == ' ' || ch == '\t' || ch == '\n' || ch == '\r') {
            ++i;
        } else if (ch == '"') {
            size_t j = i + 1;
            while (j < n && text[j] != '"') ++j;
            out.emplace_back(text.substr(i, j + 1 - i));
            i = j + 1;
        } else if (ch == '(' || ch == ')' || ch == '{' || ch == '}' || ch == '[' || ch == ']' || ch == ';') {
            out.emplace_back(1, ch);
            ++i;
        } else {
            size_t j = i;
            while (j < n) {
                const char c = text[j];
                if (c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == '(' || c == ')' || c == '{' || c == '}' ||
                    c == '[' || c == ']' || c == ';' || c == '"')
                    break;
                if (c == '/' && j + 1 < n && (text[j + 1] == '/' || text[j + 1] == '*')) break;
                ++j;
            }
            out.emplace_back(text.substr(i, j - i));
            i = j;
        }
    }
    return out;
}

bool parse_number(const std::string& tok, double* v) {
    if (tok.empty()) return false;
    char* end = nullptr;
    const double x = std::strtod(tok.c_str(), &end);
    if (end != tok.c_str() + tok.size()) return false;
    *v = x;
    return true;
}

std::string unquote(const std::string& s) {
    return s.size() >= 2 && s.front() == '"' && s.back() == '"' ? s.substr(1, s.size() - 2) : s;
}

class Parser {
public:
    Parser(const std::vector<std::string>& t, size_t i) : t_(t), i_(i) {}
    bool done() const { return i_ >= t_.size(); }
    const std::string& peek(size_t k = 0) const {
        static const std::string none;
        return i_ + k < t_.size() ? t_[i_ + k] : none;
    }
    const std::string& next() {
        if (done()) throw FoamError("unexpected end of file");
        return t_[i_++];
    }
    void expect(const std::string& s) {
        const std::string& got = next();
        if (got != s) throw FoamError("expected '" + s + "', got '" + got + "'");
    }

    FoamValue dict_body(bool to_eof) {
        FoamValue d;
        d.kind = FoamValue::Dict;
        for (;;) {
            if (done()) {
                if (to_eof) return d;
                throw FoamError("unterminated dictionary");
            }
            if (peek() == "}") {
                if (to_eof) throw FoamError("unbalanced '}'");
                next();
                return d;
            }
            const std::string key = unquote(next());
            if (peek() == "{") {
                next();
                d.entries.emplace_back(key, dict_body(false));
                continue;
            }
            std::vector<FoamValue> vals;
            while (peek() != ";") {
                if (done()) throw FoamError("entry '" + key + "' without ';'");
                vals.push_back(value());
            }
            next();
            if (vals.size() == 1) {
                d.entries.emplace_back(key, std::move(vals[0]));
            } else {
                FoamValue l;
                l.kind = FoamValue::List;
                l.items = std::move(vals);
                d.entries.emplace_back(key, std::move(l));
            }
        }
    }

    FoamValue list_body() {
        expect("(");
        FoamValue l;
        l.kind = FoamValue::List;
        while (peek() != ")") {
            if (done()) throw FoamError("unterminated list");
            l.items.push_back(value());
        }
        next();
        return l;
    }

    FoamValue value() {
        const std::string& tok = peek();
        if (tok == "(") return list_body();
        if (tok == "{") {
            next();
            return dict_body(false);
        }
        if (tok == "[") {
            next();
            FoamValue d;
            d.kind = FoamValue::Dims;
            while (peek() != "]") {
                FoamValue x;
                x.kind = FoamValue::Number;
                if (!parse_number(next(), &x.num)) throw FoamError("bad dimension set");
                d.items.push_back(x);
            }
            next();
            return d;
        }
        const std::string word = next();
        double x;
        if (parse_number(word, &x)) {
            if (peek() == "(") return list_body();   // counted list "N ( ... )"
            if (peek() == "{") {                      // uniform list "N{value}"
                next();
                FoamValue v = value();
                expect("}");
                FoamValue l;
                l.kind = FoamValue::List;
                l.items.assign(static_cast<size_t>(x), v);
                return l;
            }
            FoamValue v;
            v.kind = FoamValue::Number;
            v.num = x;
            return v;
        }
        FoamValue w;
        w.kind = FoamValue::Word;
        w.word = unquote(word);
        return w;
    }

private:
    const std::vector<std::string>& t_;
    size_t i_;
};

// tokens after the FoamFile header
std::vector<std::string> body_tokens(const std::string& path) {
    std::vector<std::string> t = tokenize(slurp(path));
    if (!t.empty() && t[0] == "FoamFile") {
        int depth = 0;
        for (size_t k = 0; k < t.size(); ++k) {
            if (t[k] == "{") ++depth;
            if (t[k] == "}" && --depth == 0) return std::vector<std::string>(t.begin() + k + 1, t.end());
        }
        throw FoamError(path + ": unterminated FoamFile header");
    }
    return t;
}

double to_num(const std::string& tok, const std::string& where) {
    double v;
    if (!parse_number(tok, &v)) throw FoamError(where + ": expected a number, got '" + tok + "'");
    return v;
}

// the numbers of a field value: a number, or a list of numbers (vector)
void append_numbers(const FoamValue& v, std::vector<double>& out) {
    if (v.kind == FoamValue::Number) {
        out.push_back(v.num);
    } else if (v.kind == FoamValue::List) {
        for (const FoamValue& x : v.items) append_numbers(x, out);
    } else {
        throw FoamError("expected a number or a list of numbers");
    }
}

// "uniform x" or "nonuniform List<T> N ( ... )" for n entries of ncomp components
std::vector<double> field_value(const FoamValue& v, int ncomp, int64_t n) {
    if (v.kind != FoamValue::List || v.items.empty() || v.items[0].kind != FoamValue::Word)
        throw FoamError("unsupported field value");
    const std::string& how = v.items[0].word;
    std::vector<double> out;
    if (how == "uniform" && v.items.size() == 2) {
        std::vector<double> one;
        append_numbers(v.items[1], one);
        if (static_cast<int>(one.size()) != ncomp) throw FoamError("uniform value with the wrong number of components");
        out.reserve(static_cast<size_t>(n) * ncomp);
        for (int64_t i = 0; i < n; ++i) out.insert(out.end(), one.begin(), one.end());
        return out;
    }
    if (how == "nonuniform") {
        append_numbers(v.items.back(), out);
        if (static_cast<int64_t>(out.size()) != n * ncomp)
            throw FoamError("nonuniform value with " + std::to_string(out.size()) + " numbers, expected " +
                            std::to_string(n * ncomp));
        return out;
    }
    throw FoamError("unsupported field value '" + how + "'");
}

void make_dirs(const std::string& path) {
    for (size_t k = 1; k <= path.size(); ++k)
        if (k == path.size() || path[k] == '/') mkdir(path.substr(0, k).c_str(), 0755);
}

// an OpenFOAM Switch entry (yes/no, on/off, true/false, y/n, t/f, none)
bool switch_value(const FoamValue& v) {
    if (v.kind != FoamValue::Word) throw FoamError("entry is not a switch");
    const std::string& w = v.word;
    if (w == "yes" || w == "on" || w == "true" || w == "y" || w == "t") return true;
    if (w == "no" || w == "off" || w == "false" || w == "n" || w == "f" || w == "none") return false;
    throw FoamError("bad switch value '" + w + "'");
}

}  // namespace

const FoamValue* FoamValue::find(const std::string& key) const {
    for (const auto& e : entries)
        if (e.first == key) return &e.second;
    return nullptr;
}

const FoamValue& FoamValue::at(const std::string& key) const {
    const FoamValue* v = find(key);
    if (!v) throw FoamError("missing entry '" + key + "'");
    return *v;
}

double FoamValue::number() const {
    if (kind == Number) return num;
    if (kind == List)
        for (auto it = items.rbegin(); it != items.rend(); ++it)
            if (it->kind == Number) return it->num;
    throw FoamError("entry is not a number");
}

FoamValue read_dict(const std::string& path) {
    const std::vector<std::string> t = tokenize(slurp(path));
    try {
        return Parser(t, 0).dict_body(true);
    } catch (const FoamError& e) {
        throw FoamError(path + ": " + e.what());
    }
}

std::vector<double> read_scalar_list(const std::string& path) {
    const std::vector<std::string> t = body_tokens(path);
    if (t.size() < 2) throw FoamError(path + ": empty list");
    const auto n = static_cast<size_t>(to_num(t[0], path));
    if (t[1] == "{") {
        if (t.size() < 4) throw FoamError(path + ": bad uniform list");
        return std::vector<double>(n, to_num(t[2], path));
    }
    if (t[1] != "(" || t.size() < n + 3 || t[n + 2] != ")") throw FoamError(path + ": bad list");
    std::vector<double> v(n);
    for (size_t k = 0; k < n; ++k) v[k] = to_num(t[k + 2], path);
    return v;
}

std::vector<int64_t> read_label_list(const std::string& path) {
    const std::vector<double> v = read_scalar_list(path);
    return std::vector<int64_t>(v.begin(), v.end());
}

std::vector<double> read_points(const std::string& path) {
    const std::vector<std::string> t = body_tokens(path);
    const auto n = static_cast<size_t>(to_num(t.at(0), path));
    std::vector<double> p;
    p.reserve(3 * n);
    size_t k = 2;
    for (size_t i = 0; i < n; ++i) {
        if (t.at(k) != "(") throw FoamError(path + ": bad point");
        for (int q = 0; q < 3; ++q) p.push_back(to_num(t.at(k + 1 + q), path));
        k += 5;
    }
    return p;
}

void read_faces(const std::string& path, std::vector<int64_t>& offsets, std::vector<int64_t>& labels) {
    const std::vector<std::string> t = body_tokens(path);
    const auto n = static_cast<size_t>(to_num(t.at(0), path));
    if (t.at(1) != "(") throw FoamError(path + ": bad face list");
    offsets.assign(1, 0);
    labels.clear();
    size_t k = 2;
    for (size_t i = 0; i < n; ++i) {
        const auto m = static_cast<size_t>(to_num(t.at(k), path));
        if (t.at(k + 1) != "(" || t.at(k + 2 + m) != ")") throw FoamError(path + ": bad face");
        for (size_t j = 0; j < m; ++j) labels.push_back(static_cast<int64_t>(to_num(t[k + 2 + j], path)));
        offsets.push_back(static_cast<int64_t>(labels.size()));
        k += m + 3;
    }
}

std::vector<PatchInfo> read_boundary(const std::string& path) {
    const std::vector<std::string> t = body_tokens(path);
    Parser p(t, 1);   // after the count
    const FoamValue l = p.list_body();
    std::vector<PatchInfo> out;
    for (size_t k = 0; k + 1 < l.items.size(); k += 2) {
        const FoamValue& d = l.items[k + 1];
        if (l.items[k].kind != FoamValue::Word || d.kind != FoamValue::Dict) throw FoamError(path + ": bad patch entry");
        PatchInfo pi;
        pi.name = l.items[k].word;
        pi.type = d.at("type").word;
        pi.size = static_cast<int64_t>(d.at("nFaces").number());
        pi.start = static_cast<int64_t>(d.at("startFace").number());
        out.push_back(pi);
    }
    return out;
}

PolyMesh read_polymesh(const std::string& case_dir, const std::string& mesh) {
    const std::string base = case_dir + "/constant/" + mesh + "/";
    PolyMesh m;
    m.points = read_points(base + "points");
    read_faces(base + "faces", m.face_offsets, m.face_points);
    m.owner = read_label_list(base + "owner");
    m.neighbour = read_label_list(base + "neighbour");
    m.patches = read_boundary(base + "boundary");
    int64_t mx = -1;
    for (int64_t o : m.owner) mx = std::max(mx, o);
    for (int64_t o : m.neighbour) mx = std::max(mx, o);
    m.n_cells = mx + 1;
    int empty = 0;
    for (const PatchInfo& p : m.patches) empty += (p.type == "empty" && p.size > 0) ? 1 : 0;
    m.n_solution_dims = 3 - empty;
    if (m.n_faces() + 1 != static_cast<int64_t>(m.face_offsets.size()))
        throw FoamError(base + ": owner and faces disagree on the face count");
    return m;
}

VolField read_vol_field(const std::string& path, int64_t n_cells, const std::vector<PatchInfo>& patches) {
    const FoamValue d = read_dict(path);
    VolField f;
    const FoamValue* hdr = d.find("FoamFile");
    const FoamValue* cls = hdr ? hdr->find("class") : nullptr;
    f.ncomp = (cls && cls->word == "volVectorField") ? 3 : 1;
    try {
        f.internal = field_value(d.at("internalField"), f.ncomp, n_cells);
        const FoamValue& bf = d.at("boundaryField");
        for (const auto& e : bf.entries) {
            VolField::Patch p;
            p.type = e.second.at("type").word;
            int64_t size = 0;
            for (const PatchInfo& pi : patches)
                if (pi.name == e.first) size = pi.size;
            if (const FoamValue* v = e.second.find("value")) p.value = field_value(*v, f.ncomp, size);
            if (const FoamValue* v = e.second.find("pressureIn")) p.pressure = v->number();
            if (const FoamValue* v = e.second.find("pressureOut")) p.pressure = v->number();
            f.patches[e.first] = p;
        }
    } catch (const FoamError& e) {
        throw FoamError(path + ": " + e.what());
    }
    return f;
}

Case read_case(const std::string& dir, bool vmesh) {
    Case c;
    c.dir = dir;
    c.mesh = read_polymesh(dir);
    c.D = c.mesh.n_solution_dims;
    c.xis = read_scalar_list(dir + "/constant/Xis");
    c.weights = read_scalar_list(dir + "/constant/weights");
    if (c.xis.size() != c.weights.size()) throw FoamError("constant/Xis and constant/weights differ in length");
    const FoamValue props = read_dict(dir + "/constant/DVMProperties");
    const FoamValue& gp = props.at("gasProperties");
    const FoamValue& fp = props.at("fvDVMparas");
    c.R = gp.at("R").number();
    c.omega = gp.at("omega").number();
    c.Tref = gp.at("Tref").number();
    c.mu_ref = gp.at("muRef").number();
    c.Pr = gp.at("Pr").number();
    c.K_inner = gp.find("KInner") ? static_cast<int>(gp.at("KInner").number()) : 0;   // fvDVM.C:1948
    c.xi_max = fp.at("xiMax").number();
    if (vmesh) {
        // the velocity mesh's cell centres and volumes, xiMax = max |xi|
        // (fvDVM.C:166-196; 2-D drops z)
        const PolyMesh vm = read_polymesh(dir, "vMesh");
        const int64_t nF = vm.n_faces(), nv = vm.n_cells;
        std::vector<double> Cf(3 * nF), Sf(3 * nF), C(3 * nv), V(nv);
        const int st = dugks_mesh_geometry(static_cast<int32_t>(vm.points.size() / 3), vm.points.data(),
                                           static_cast<int32_t>(nF), vm.face_offsets.data(), vm.face_points.data(),
                                           vm.owner.data(), static_cast<int32_t>(vm.n_internal()),
                                           vm.neighbour.data(), static_cast<int32_t>(nv), Cf.data(), Sf.data(),
                                           C.data(), V.data());
        if (st != DUGKS_OK) throw FoamError("constant/vMesh: geometry failed");
        c.xi_max = 0;
        for (int64_t i = 0; i < nv; ++i) {
            if (c.D == 2) C[3 * i + 2] = 0.0;
            c.xi_max = std::max(c.xi_max, std::sqrt(C[3 * i] * C[3 * i] + C[3 * i + 1] * C[3 * i + 1] +
                                                    C[3 * i + 2] * C[3 * i + 2]));
        }
        c.dv_xi = C;
        c.dv_w = V;
    }
    if (const FoamValue* mf = fp.find("macroFlux")) c.macro_flux = mf->kind == FoamValue::Word && mf->word == "yes";
    const int64_t nc = c.mesh.n_cells;
    const VolField rho = read_vol_field(dir + "/0/rho", nc, c.mesh.patches);
    const VolField U = read_vol_field(dir + "/0/U", nc, c.mesh.patches);
    const VolField T = read_vol_field(dir + "/0/T", nc, c.mesh.patches);
    if (U.ncomp != 3 || rho.ncomp != 1 || T.ncomp != 1) throw FoamError("0/rho, 0/U, 0/T: wrong field classes");
    c.rho0 = rho.internal;
    c.U0 = U.internal;
    c.T0 = T.internal;
    for (const PatchInfo& p : c.mesh.patches) {
        auto rt = rho.patches.find(p.name);
        // constraint (empty) patches need no field entry
        const std::string type = rt != rho.patches.end() ? rt->second.type : p.type;
        static const std::map<std::string, PatchKind> by_type = {
            {"empty", PatchKind::Empty},
            {"calculatedMaxwell", PatchKind::MaxwellWall},
            {"farField", PatchKind::FarField},
            {"zeroGradient", PatchKind::ZeroGradient},
            {"fixedValue", PatchKind::Mixed},
            {"symmetryPlane", PatchKind::Symmetry},
            {"symmetryMod", PatchKind::DVMSymmetry},
            {"pressureIn", PatchKind::PressureIn},
            {"pressureOut", PatchKind::PressureOut}};
        const auto kt = by_type.find(type);
        if (kt == by_type.end()) throw FoamError("patch " + p.name + ": rho patch type '" + type + "' is not supported");
        const PatchKind kind = kt->second;
        c.kinds.push_back(kind);
        c.patch_p.push_back(rt != rho.patches.end() ? rt->second.pressure : 0.0);
        auto first = [&](const VolField& f, int comp, double dflt) {
            auto it = f.patches.find(p.name);
            if (it == f.patches.end() || it->second.value.empty()) return dflt;
            return it->second.value[comp];
        };
        auto type_of = [&](const VolField& f) {
            auto it = f.patches.find(p.name);
            return it == f.patches.end() ? p.type : it->second.type;
        };
        c.rho_types.push_back(type);
        c.U_types.push_back(type_of(U));
        c.T_types.push_back(type_of(T));
        c.patch_rho.push_back(first(rho, 0, 0.0));
        for (int q = 0; q < 3; ++q) c.patch_U.push_back(first(U, q, 0.0));
        c.patch_T.push_back(first(T, 0, c.Tref));
    }
    std::ifstream cd(dir + "/system/controlDict");
    if (cd) {
        const FoamValue d = read_dict(dir + "/system/controlDict");
        if (const FoamValue* v = d.find("startTime")) c.start_time = v->number();
        if (const FoamValue* v = d.find("endTime")) c.end_time = v->number();
        if (const FoamValue* v = d.find("deltaT")) c.delta_t = v->number();
        if (const FoamValue* v = d.find("writeInterval")) c.write_interval = v->number();
        if (const FoamValue* v = d.find("adjustTimeStep")) c.adjust_time_step = switch_value(*v);
        if (const FoamValue* v = d.find("maxCo")) c.max_co = v->number();
        if (const FoamValue* v = d.find("maxDeltaT")) c.max_delta_t = v->number();
    }
    return c;
}

int32_t patch_type_of(PatchKind k) {
    switch (k) {
        case PatchKind::MaxwellWall: return DUGKS_PATCH_MAXWELL_WALL;
        case PatchKind::FarField: return DUGKS_PATCH_FAR_FIELD;
        case PatchKind::ZeroGradient: return DUGKS_PATCH_ZERO_GRADIENT;
        case PatchKind::Mixed: return DUGKS_PATCH_MIXED;
        case PatchKind::Symmetry: return DUGKS_PATCH_SYMMETRY;
        case PatchKind::DVMSymmetry: return DUGKS_PATCH_DVM_SYMMETRY;
        case PatchKind::PressureIn: return DUGKS_PATCH_PRESSURE_IN;
        case PatchKind::PressureOut: return DUGKS_PATCH_PRESSURE_OUT;
        default: return 0;
    }
}

const char* kind_name(PatchKind k) {
    switch (k) {
        case PatchKind::Empty: return "empty";
        case PatchKind::MaxwellWall: return "maxwellWall";
        case PatchKind::FarField: return "farField";
        case PatchKind::ZeroGradient: return "zeroGradient";
        case PatchKind::Mixed: return "mixed";
        case PatchKind::Symmetry: return "symmetryPlane";
        case PatchKind::DVMSymmetry: return "DVMsymmetry";
        case PatchKind::PressureIn: return "pressureIn";
        default: return "pressureOut";
    }
}

FlatMesh flatten(const Case& c) {
    const PolyMesh& pm = c.mesh;
    const int64_t nF = pm.n_faces(), nIF = pm.n_internal(), nC = pm.n_cells;
    std::vector<double> Cf(3 * nF), Sf(3 * nF), C(3 * nC), V(nC);
    const int st = dugks_mesh_geometry(static_cast<int32_t>(pm.points.size() / 3), pm.points.data(),
                                       static_cast<int32_t>(nF), pm.face_offsets.data(), pm.face_points.data(),
                                       pm.owner.data(), static_cast<int32_t>(nIF), pm.neighbour.data(),
                                       static_cast<int32_t>(nC), Cf.data(), Sf.data(), C.data(), V.data());
    if (st != DUGKS_OK) throw FoamError("dugks_mesh_geometry failed with status " + std::to_string(st));
    FlatMesh f;
    f.n_cells = static_cast<int32_t>(nC);
    f.n_internal = static_cast<int32_t>(nIF);
    f.D = c.D;
    f.C = C;
    f.V = V;
    f.neighbour = pm.neighbour;
    f.owner.assign(pm.owner.begin(), pm.owner.begin() + nIF);
    f.Cf.assign(Cf.begin(), Cf.begin() + 3 * nIF);
    f.Sf.assign(Sf.begin(), Sf.begin() + 3 * nIF);
    f.patch_start.push_back(0);
    for (size_t p = 0; p < pm.patches.size(); ++p) {
        const PatchInfo& pi = pm.patches[p];
        if (c.kinds[p] == PatchKind::Empty) {
            if (pi.size > 0 && pm.n_solution_dims == 3) throw FoamError("empty patch on a 3-D mesh");
            continue;
        }
        for (int64_t k = pi.start; k < pi.start + pi.size; ++k) {
            f.owner.push_back(pm.owner[k]);
            f.Cf.insert(f.Cf.end(), Cf.begin() + 3 * k, Cf.begin() + 3 * k + 3);
            f.Sf.insert(f.Sf.end(), Sf.begin() + 3 * k, Sf.begin() + 3 * k + 3);
            // pressureIn/Out and symmetryMod rho patches start at one: their
            // dictionary constructors read no value and assign pTraits::one
            // (pressureInFvPatchField.C:72-75, symmetryModFvPatchField.C:72)
            const bool at_one = c.kinds[p] == PatchKind::PressureIn || c.kinds[p] == PatchKind::PressureOut ||
                                c.kinds[p] == PatchKind::DVMSymmetry;
            f.rho_b.push_back(at_one ? 1.0 : c.patch_rho[p]);
            f.U_b.insert(f.U_b.end(), c.patch_U.begin() + 3 * p, c.patch_U.begin() + 3 * p + 3);
            f.T_b.push_back(c.patch_T[p]);
            f.p_b.push_back(c.patch_p[p]);
        }
        f.patch_type.push_back(patch_type_of(c.kinds[p]));
        f.patch_start.push_back(f.patch_start.back() + static_cast<int32_t>(pi.size));
        f.patch_of.push_back(static_cast<int>(p));
    }
    f.n_boundary = f.patch_start.back();
    return f;
}

void write_vol_field(const std::string& path, const std::string& name, int ncomp, const std::vector<double>& internal,
                     const std::vector<std::pair<std::string, std::pair<std::string, std::vector<double>>>>& patches,
                     const std::string& dims, const std::string& location) {
    const size_t slash = path.rfind('/');
    if (slash != std::string::npos) make_dirs(path.substr(0, slash));
    std::FILE* f = std::fopen(path.c_str(), "w");
    if (!f) throw FoamError("cannot write " + path);
    const bool vec = ncomp == 3;
    const char* T = vec ? "vector" : "scalar";
    auto put = [&](const double* v) {
        if (vec) std::fprintf(f, "(%.15g %.15g %.15g)", v[0], v[1], v[2]);
        else std::fprintf(f, "%.15g", v[0]);
    };
    std::fprintf(f,
                 "FoamFile\n{\n    version     2.0;\n    format      ascii;\n    class       %s;\n"
                 "    location    \"%s\";\n    object      %s;\n}\n\ndimensions      %s;\n\n",
                 vec ? "volVectorField" : "volScalarField", location.c_str(), name.c_str(), dims.c_str());
    const size_t n = internal.size() / ncomp;
    std::fprintf(f, "internalField   nonuniform List<%s>\n%zu\n(\n", T, n);
    for (size_t i = 0; i < n; ++i) {
        put(&internal[i * ncomp]);
        std::fputc('\n', f);
    }
    std::fprintf(f, ")\n;\n\nboundaryField\n{\n");
    for (const auto& p : patches) {
        std::fprintf(f, "    %s\n    {\n        type            %s;\n", p.first.c_str(), p.second.first.c_str());
        const std::vector<double>& v = p.second.second;
        if (!v.empty()) {
            const size_t m = v.size() / ncomp;
            std::fprintf(f, "        value           nonuniform List<%s> %zu(", T, m);
            for (size_t i = 0; i < m; ++i) {
                if (i) std::fputc(' ', f);
                put(&v[i * ncomp]);
            }
            std::fprintf(f, ");\n");
        }
        std::fprintf(f, "    }\n");
    }
    std::fprintf(f, "}\n");
    if (std::fclose(f) != 0) throw FoamError("error writing " + path);
}

std::string time_name(double t) {
    char buf[64];
    std::snprintf(buf, sizeof buf, "%g", t);
    return buf;
}

}  // namespace dugks_host
