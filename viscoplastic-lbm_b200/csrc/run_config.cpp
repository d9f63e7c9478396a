// run_config.cpp -- the run configuration of the drop-in driver, read from the
// YAML file the reference's configuration tool reads (pyvisc:
// conf_handler.read_configs, pyvisc/conf_handler.py:15-24, validated by
// SchemeVarH, pyvisc/schemes.py:53-74; example examples/all_options.yaml).
//
// The file is a YAML sequence whose first item is a mapping of the SchemeVarH
// keys (a bare mapping is accepted too).  The keys map onto the compile-time
// constants pyvisc renders into var.h (pyvisc/templates/var.h.j2) and from
// there onto vlbm_config / vlbm_run_config.  Keys pyvisc does not know are the
// extension keys listed in include/vlbm.h; other unknown keys are ignored, as
// pydantic ignores them.  The parser reads the YAML subset such files use:
// block mappings and sequences by indentation, flow sequences [a, b],
// scalars (plain, single- or double-quoted), comments.
#include <cctype>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <utility>
#include <vector>
#include "internal.h"

namespace {

struct Node {
    enum Kind { NUL, SCALAR, MAP, SEQ } kind = NUL;
    std::string s;
    bool quoted = false;
    std::vector<std::pair<std::string, Node>> map;
    std::vector<Node> seq;
    int line = 0;
    const Node* get(const char* k) const {
        for (auto& kv : map)
            if (kv.first == k) return &kv.second;
        return nullptr;
    }
};

struct Line {
    int indent;
    std::string text;   // without indentation and comment
    int no;
};

struct ParseError {
    std::string msg;
    bool unsupported = false;   // a valid value this library does not run
};

std::string strip_comment(const std::string& s) {
    bool sq = false, dq = false;
    for (size_t i = 0; i < s.size(); ++i) {
        const char c = s[i];
        if (c == '\'' && !dq) sq = !sq;
        else if (c == '"' && !sq) dq = !dq;
        else if (c == '#' && !sq && !dq && (i == 0 || std::isspace((unsigned char)s[i - 1]))) return s.substr(0, i);
    }
    return s;
}

std::string rtrim(std::string s) {
    while (!s.empty() && std::isspace((unsigned char)s.back())) s.pop_back();
    return s;
}
std::string trim(const std::string& s) {
    size_t a = 0;
    while (a < s.size() && std::isspace((unsigned char)s[a])) ++a;
    return rtrim(s.substr(a));
}

Node scalar(const std::string& raw, int line) {
    Node n;
    n.line = line;
    std::string t = trim(raw);
    if (t.size() >= 2 && ((t.front() == '"' && t.back() == '"') || (t.front() == '\'' && t.back() == '\''))) {
        n.kind = Node::SCALAR;
        n.quoted = true;
        n.s = t.substr(1, t.size() - 2);
        return n;
    }
    if (t.empty() || t == "~" || t == "null" || t == "Null" || t == "NULL") {
        n.kind = Node::NUL;
        return n;
    }
    n.kind = Node::SCALAR;
    n.s = t;
    return n;
}

// Flow sequence "[a, b, [c, d]]".
Node flow_seq(const std::string& t, size_t& i, int line) {
    Node n;
    n.kind = Node::SEQ;
    n.line = line;
    ++i;   // '['
    std::string cur;
    bool sq = false, dq = false;
    auto flush = [&]() {
        std::string v = trim(cur);
        if (!v.empty()) n.seq.push_back(scalar(v, line));
        cur.clear();
    };
    while (i < t.size()) {
        const char c = t[i];
        if (!sq && !dq && c == '[') {
            n.seq.push_back(flow_seq(t, i, line));
            cur.clear();
            continue;
        }
        if (c == '\'' && !dq) sq = !sq;
        if (c == '"' && !sq) dq = !dq;
        if (!sq && !dq && c == ']') {
            flush();
            ++i;
            return n;
        }
        if (!sq && !dq && c == ',') {
            flush();
            ++i;
            continue;
        }
        cur.push_back(c);
        ++i;
    }
    throw ParseError{"line " + std::to_string(line) + ": unterminated flow sequence"};
}

Node value_of(const std::string& raw, int line) {
    const std::string t = trim(raw);
    if (!t.empty() && t[0] == '[') {
        size_t i = 0;
        Node n = flow_seq(t, i, line);
        if (!trim(t.substr(i)).empty()) throw ParseError{"line " + std::to_string(line) + ": text after ']'"};
        return n;
    }
    if (!t.empty() && t[0] == '{') throw ParseError{"line " + std::to_string(line) + ": flow mappings are not supported"};
    return scalar(t, line);
}

// Position of the ':' that ends a mapping key ("key: value" or "key:").
size_t key_colon(const std::string& t) {
    bool sq = false, dq = false;
    for (size_t i = 0; i < t.size(); ++i) {
        const char c = t[i];
        if (c == '\'' && !dq) sq = !sq;
        else if (c == '"' && !sq) dq = !dq;
        else if (c == ':' && !sq && !dq && (i + 1 == t.size() || t[i + 1] == ' ')) return i;
    }
    return std::string::npos;
}

struct Parser {
    std::vector<Line> lines;
    size_t pos = 0;

    Node block(int indent) {
        if (pos >= lines.size() || lines[pos].indent < indent) return Node{};
        const Line& first = lines[pos];
        if (first.text[0] == '-' && (first.text.size() == 1 || first.text[1] == ' ')) return seq(first.indent);
        return mapping(first.indent);
    }

    Node seq(int indent) {
        Node n;
        n.kind = Node::SEQ;
        n.line = lines[pos].no;
        while (pos < lines.size() && lines[pos].indent == indent && lines[pos].text[0] == '-' &&
               (lines[pos].text.size() == 1 || lines[pos].text[1] == ' ')) {
            Line& l = lines[pos];
            std::string rest = l.text.size() > 1 ? l.text.substr(2) : std::string();
            size_t lead = 0;
            while (lead < rest.size() && rest[lead] == ' ') ++lead;
            rest = rest.substr(lead);
            if (rest.empty()) {
                ++pos;
                n.seq.push_back(block(indent + 1));
            } else if (rest[0] != '[' && key_colon(rest) != std::string::npos) {
                // "- key: value": a mapping whose keys sit at the column of "key"
                l.indent = indent + 2 + (int)lead;
                l.text = rest;
                n.seq.push_back(mapping(l.indent));
            } else {
                ++pos;
                n.seq.push_back(value_of(rest, l.no));
            }
        }
        if (pos < lines.size() && lines[pos].indent > indent)
            throw ParseError{"line " + std::to_string(lines[pos].no) + ": bad indentation"};
        return n;
    }

    Node mapping(int indent) {
        Node n;
        n.kind = Node::MAP;
        n.line = lines[pos].no;
        while (pos < lines.size() && lines[pos].indent == indent) {
            const Line& l = lines[pos];
            if (l.text[0] == '-' && (l.text.size() == 1 || l.text[1] == ' '))
                throw ParseError{"line " + std::to_string(l.no) + ": sequence item inside a mapping"};
            const size_t c = key_colon(l.text);
            if (c == std::string::npos) throw ParseError{"line " + std::to_string(l.no) + ": expected 'key: value'"};
            std::string key = trim(l.text.substr(0, c));
            if (key.size() >= 2 && (key.front() == '"' || key.front() == '\'')) key = key.substr(1, key.size() - 2);
            const std::string rest = trim(l.text.substr(c + 1));
            for (auto& kv : n.map)
                if (kv.first == key) throw ParseError{"line " + std::to_string(l.no) + ": duplicate key '" + key + "'"};
            ++pos;
            if (!rest.empty()) {
                n.map.emplace_back(key, value_of(rest, l.no));
            } else if (pos < lines.size() && (lines[pos].indent > indent ||
                                              (lines[pos].indent == indent && lines[pos].text[0] == '-'))) {
                // block value; a sequence may sit at the key's own column
                n.map.emplace_back(key, block(lines[pos].indent));
            } else {
                Node nul;
                nul.line = l.no;
                n.map.emplace_back(key, nul);
            }
        }
        if (pos < lines.size() && lines[pos].indent > indent)
            throw ParseError{"line " + std::to_string(lines[pos].no) + ": bad indentation"};
        return n;
    }
};

Node parse_yaml(const std::string& text) {
    Parser p;
    int no = 0;
    size_t a = 0;
    while (a <= text.size()) {
        size_t b = text.find('\n', a);
        if (b == std::string::npos) b = text.size();
        std::string raw = text.substr(a, b - a);
        ++no;
        a = b + 1;
        if (!raw.empty() && raw.back() == '\r') raw.pop_back();
        if (raw.find('\t') != std::string::npos && raw.find_first_not_of(" \t") != std::string::npos &&
            raw.find('\t') < raw.find_first_not_of(" \t"))
            throw ParseError{"line " + std::to_string(no) + ": tab in indentation"};
        std::string s = rtrim(strip_comment(raw));
        if (trim(s).empty()) continue;
        if (trim(s) == "---" || trim(s) == "...") continue;
        int ind = 0;
        while (ind < (int)s.size() && s[ind] == ' ') ++ind;
        p.lines.push_back({ind, s.substr(ind), no});
    }
    if (p.lines.empty()) throw ParseError{"empty document"};
    Node root = p.block(p.lines[0].indent);
    if (p.pos != p.lines.size()) throw ParseError{"line " + std::to_string(p.lines[p.pos].no) + ": bad indentation"};
    return root;
}

// ---------------------------------------------------------------- typing --
struct Reader {
    const Node* map;
    std::string where;

    [[noreturn]] void fail(const std::string& key, const std::string& why, const Node* n = nullptr) const {
        throw ParseError{where + key + (n ? " (line " + std::to_string(n->line) + ")" : std::string()) + ": " + why};
    }
    const Node* req(const char* k) const {
        const Node* n = map->get(k);
        if (!n) fail(k, "field required");
        return n;
    }
    static bool is_int(const std::string& s) {
        if (s.empty()) return false;
        size_t i = (s[0] == '-' || s[0] == '+') ? 1 : 0;
        if (i == s.size()) return false;
        for (; i < s.size(); ++i)
            if (!std::isdigit((unsigned char)s[i]) && s[i] != '_') return false;
        return true;
    }
    long long as_int(const char* k, const Node* n) const {
        if (n->kind != Node::SCALAR || n->quoted || !is_int(n->s)) fail(k, "value is not a valid integer", n);
        std::string t;
        for (char c : n->s)
            if (c != '_') t.push_back(c);
        errno = 0;
        const long long v = std::strtoll(t.c_str(), nullptr, 10);
        if (errno) fail(k, "integer out of range", n);
        return v;
    }
    double as_float(const char* k, const Node* n) const {
        if (n->kind != Node::SCALAR || n->quoted) fail(k, "value is not a valid float", n);
        std::string t = n->s;
        if (t == ".inf" || t == ".Inf" || t == "+.inf") return INFINITY;
        if (t == "-.inf" || t == "-.Inf") return -INFINITY;
        if (t == ".nan" || t == ".NaN") return NAN;
        char* end = nullptr;
        errno = 0;
        const double v = std::strtod(t.c_str(), &end);
        if (end == t.c_str() || *end != '\0' || errno == ERANGE) fail(k, "value is not a valid float", n);
        return v;
    }
    bool as_bool(const char* k, const Node* n) const {
        if (n->kind == Node::SCALAR && !n->quoted) {
            const std::string& t = n->s;
            if (t == "true" || t == "True" || t == "TRUE") return true;
            if (t == "false" || t == "False" || t == "FALSE") return false;
            if (t == "1") return true;
            if (t == "0") return false;
        }
        fail(k, "value could not be parsed to a boolean", n);
    }
    std::string as_str(const char* k, const Node* n) const {
        if (n->kind != Node::SCALAR) fail(k, "str type expected", n);
        return n->s;
    }
    // optional getters
    bool has(const char* k) const { return map->get(k) != nullptr; }
    long long i(const char* k, long long d) const { const Node* n = map->get(k); return n ? as_int(k, n) : d; }
    double f(const char* k, double d) const { const Node* n = map->get(k); return n ? as_float(k, n) : d; }
    bool b(const char* k, bool d) const { const Node* n = map->get(k); return n ? as_bool(k, n) : d; }
    void vec(const char* k, double* out, int len) const {
        const Node* n = map->get(k);
        if (!n) return;
        if (n->kind != Node::SEQ || (int)n->seq.size() > len) fail(k, "expected a list of at most " + std::to_string(len) + " numbers", n);
        for (size_t j = 0; j < n->seq.size(); ++j) out[j] = as_float(k, &n->seq[j]);
    }
};

const char* const kBuilderNames[] = {"periodic",      "plates_y",          "lid_driven",     "closed_box",
                                     "square_duct",   "duct_yz",           "lid_cavity_closed",
                                     "plates_y_free_slip", "plates_y_zouhe", "circular_duct", "annular_duct"};

void copy_str(char* dst, size_t cap, const std::string& s, const char* key) {
    if (s.size() + 1 > cap) throw ParseError{std::string(key) + ": longer than " + std::to_string(cap - 1) + " characters"};
    std::memcpy(dst, s.c_str(), s.size() + 1);
}

void fill(const Node& root, vlbm_run_config* rc, vlbm_sphere* spheres, int32_t max_spheres) {
    const Node* doc = &root;
    if (root.kind == Node::SEQ) {   // read_configs takes the first item (conf_handler.py:20)
        if (root.seq.empty()) throw ParseError{"the configuration list is empty"};
        doc = &root.seq[0];
    }
    if (doc->kind != Node::MAP) throw ParseError{"the configuration is not a mapping of keys"};
    Reader r{doc, ""};
    vlbm_config& c = rc->cfg;

    // SchemeVarH (pyvisc/schemes.py:53-74): required keys
    const std::string prec = r.as_str("precision", r.req("precision"));
    if (prec != "single" && prec != "double") r.fail("precision", "unexpected value; permitted: 'single', 'double'");
    rc->precision_double = prec == "double";
    c.nx = (int32_t)r.as_int("NX", r.req("NX"));
    c.ny = (int32_t)r.as_int("NY", r.req("NY"));
    const long long nz_gpu = r.as_int("NZ", r.req("NZ"));
    c.tau = r.as_float("tau", r.req("tau"));
    const std::string vs = r.as_str("vel_set", r.req("vel_set"));
    if (vs != "D3Q19" && vs != "D3Q27") r.fail("vel_set", "unexpected value; permitted: 'D3Q19', 'D3Q27'");
    c.vel_set = vs == "D3Q19" ? VLBM_D3Q19 : VLBM_D3Q27;
    rc->use_ibm = r.as_bool("use_ibm", r.req("use_ibm"));
    {
        const Node* n = doc->get("non_newtonian_model");
        c.rheology = VLBM_NEWTONIAN;
        if (n && n->kind != Node::NUL) {
            const std::string m = r.as_str("non_newtonian_model", n);
            if (m == "BINGHAM") c.rheology = VLBM_BINGHAM;
            else if (m == "POWERLAW") c.rheology = VLBM_POWERLAW;
            else r.fail("non_newtonian_model", "expected null, 'BINGHAM' or 'POWERLAW' (var.h:26-27)", n);
        }
    }
    const long long sim_id = r.as_int("sim_id", r.req("sim_id"));
    char idbuf[32];
    std::snprintf(idbuf, sizeof(idbuf), "%03lld", sim_id);   // var.h.j2: '%03d' % sim_id
    copy_str(rc->sim_id, sizeof(rc->sim_id), idbuf, "sim_id");
    copy_str(rc->path_save, sizeof(rc->path_save), r.as_str("path_save", r.req("path_save")), "path_save");
    rc->steps = r.as_int("steps", r.req("steps"));
    rc->macr_save = r.as_int("macr_save", r.req("macr_save"));
    rc->data_report = r.as_int("data_report", r.req("data_report"));
    // optional keys with SchemeVarH's defaults
    c.fx = r.f("FX", 0.0);
    c.fy = r.f("FY", 0.0);
    c.fz = r.f("FZ", 0.0);
    rc->data_stop = r.b("data_stop", false);
    rc->data_save = r.b("data_save", false);
    rc->pop_save = r.b("pop_save", false);
    rc->ini_step = r.i("ini_step", 0);
    rc->n_gpus = (int32_t)r.i("n_gpus", 1);
    rc->resid_max = r.f("resid_max", 1e-5);
    c.nz = (int32_t)(nz_gpu * rc->n_gpus);   // var.h: NZ_TOTAL = NZ * N_GPUS

    // extension keys (the other compile-time constants of var.h, nnf.h, ibmVar.h)
    c.rho0 = r.f("rho_0", c.rho0);
    rc->u_max = r.f("u_max", 0.1);
    {   // UX_BC..RHO_BC default to var.h:114-117 with U_MAX and RHO_0
        const double u = rc->u_max;
        const double ux[8] = {0, u, 0, 0, 0, 0, 0, 0}, uy[8] = {0, u / 2, -u / 2, 0, 0, 0, 0, 0},
                     uz[8] = {0, u, -u, 0, 0, 0, 0, 0};
        for (int k = 0; k < 8; ++k) {
            c.ux_bc[k] = ux[k]; c.uy_bc[k] = uy[k]; c.uz_bc[k] = uz[k]; c.rho_bc[k] = k == 0 ? c.rho0 : 1.0;
        }
        r.vec("ux_bc", c.ux_bc, 8);
        r.vec("uy_bc", c.uy_bc, 8);
        r.vec("uz_bc", c.uz_bc, 8);
        r.vec("rho_bc", c.rho_bc, 8);
    }
    if (r.has("collision")) {
        const std::string op = r.as_str("collision", r.req("collision"));
        if (op == "regularized") c.collision = VLBM_OP_REGULARIZED;
        else if (op == "bgk") c.collision = VLBM_OP_BGK;
        else r.fail("collision", "expected 'regularized' or 'bgk'");
    }
    c.eta_p = r.f("eta_p", c.eta_p);
    c.yield_stress = r.f("yield_stress", c.yield_stress);
    c.n_index = r.f("n_index", c.n_index);
    c.k_consistency = r.f("k_consistency", c.rho0 * (c.tau - 0.5) / 3.0);   // nnf.h:12 with this TAU
    c.gamma0 = r.f("gamma_0", c.gamma0);
    if (r.has("storage")) {
        const std::string st = r.as_str("storage", r.req("storage"));
        if (st == "f32") c.storage = VLBM_STORE_F32;
        else if (st == "f16") c.storage = VLBM_STORE_F16;
        else if (st == "bf16") c.storage = VLBM_STORE_BF16;
        else r.fail("storage", "expected 'f32', 'f16' or 'bf16'");
    }
    c.device = (int32_t)r.i("device", 0);
    rc->builder = VLBM_BUILDER_CLOSED_BOX;   // the builder file compiled by default (src/CUDA/closedBoxBounceBack.cu)
    if (r.has("builder")) {
        const std::string b = r.as_str("builder", r.req("builder"));
        int found = -1;
        for (int k = 0; k < (int)(sizeof(kBuilderNames) / sizeof(kBuilderNames[0])); ++k)
            if (b == kBuilderNames[k]) found = k;
        if (found < 0) r.fail("builder", "unknown builder '" + b + "'");
        rc->builder = found;
    }
    c.duct_outer_radius = r.f("outer_radius", 0.0);
    c.duct_inner_radius = r.f("inner_radius", 0.0);
    c.duct_outer_velocity = r.f("outer_velocity", 0.0);
    c.duct_outer_rotation = r.f("outer_rotation", 0.0);
    c.duct_inner_velocity = r.f("inner_velocity", 0.0);
    c.duct_inner_rotation = r.f("inner_rotation", 0.0);
    rc->checkpoint_save = r.i("checkpoint_save", 0);
    rc->load_checkpoint = r.b("load_checkpoint", false);
    copy_str(rc->load_folder, sizeof(rc->load_folder),
             doc->get("checkpoint_folder") ? r.as_str("checkpoint_folder", doc->get("checkpoint_folder"))
                                           : std::string(rc->path_save),
             "checkpoint_folder");

    // IBM (ibmVar.h, ibmBoundaryCondition.h) under the key `ibm`
    rc->n_spheres = 0;
    rc->particles_save = 0;
    rc->particles_nodes_save = 1;
    rc->export_forces = 0;
    if (const Node* ib = doc->get("ibm")) {
        if (ib->kind != Node::MAP) r.fail("ibm", "expected a mapping", ib);
        Reader q{ib, "ibm."};
        vlbm_ibm_config& g = rc->ibm;
        g.max_iterations = (int32_t)q.i("max_iterations", g.max_iterations);
        if (q.has("stencil")) g.stencil = (int32_t)q.i("stencil", g.stencil);
        g.thickness = q.f("thickness", g.thickness);
        g.movement_alpha = q.f("movement_discretization", g.movement_alpha);
        g.fluid_density = q.f("fluid_density", g.fluid_density);
        g.gx = q.f("gx", g.gx);
        g.gy = q.f("gy", g.gy);
        g.gz = q.f("gz", g.gz);
        g.wall_x = q.b("wall_x", g.wall_x) ? 1 : 0;
        g.wall_y = q.b("wall_y", g.wall_y) ? 1 : 0;
        g.wall_z = q.b("wall_z", g.wall_z) ? 1 : 0;
        g.pp_friction = q.f("pp_friction", g.pp_friction);
        g.pw_friction = q.f("pw_friction", g.pw_friction);
        g.pp_restitution = q.f("pp_restitution", g.pp_restitution);
        g.pw_restitution = q.f("pw_restitution", g.pw_restitution);
        g.particle_young = q.f("particle_young", g.particle_young);
        g.particle_poisson = q.f("particle_poisson", g.particle_poisson);
        g.wall_young = q.f("wall_young", g.wall_young);
        g.wall_poisson = q.f("wall_poisson", g.wall_poisson);
        g.mesh_scale = q.f("mesh_scale", g.mesh_scale);
        g.breugem = q.f("breugem", g.breugem);
        rc->particles_save = q.i("particles_save", 0);
        rc->particles_nodes_save = q.b("particles_nodes_save", true) ? 1 : 0;
        rc->export_forces = q.b("export_forces", false) ? 1 : 0;
        if (const Node* sl = ib->get("spheres")) {
            if (sl->kind != Node::SEQ) q.fail("spheres", "expected a list", sl);
            const double density = q.f("particle_density", 2.0);
            for (const Node& s : sl->seq) {
                if (s.kind != Node::MAP) q.fail("spheres", "each sphere is a mapping", &s);
                Reader t{&s, "ibm.spheres[" + std::to_string(rc->n_spheres) + "]."};
                vlbm_sphere sp;
                std::memset(&sp, 0, sizeof(sp));
                sp.diameter = t.as_float("diameter", t.req("diameter"));
                double ctr[3] = {0, 0, 0}, vel[3] = {0, 0, 0}, w[3] = {0, 0, 0};
                const Node* cn = t.req("center");
                if (cn->kind != Node::SEQ || cn->seq.size() != 3) t.fail("center", "expected [x, y, z]", cn);
                t.vec("center", ctr, 3);
                t.vec("velocity", vel, 3);
                t.vec("angular_velocity", w, 3);
                sp.cx = ctr[0]; sp.cy = ctr[1]; sp.cz = ctr[2];
                sp.vx = vel[0]; sp.vy = vel[1]; sp.vz = vel[2];
                sp.wx = w[0]; sp.wy = w[1]; sp.wz = w[2];
                sp.density = t.f("density", density);
                sp.movable = t.b("movable", true) ? 1 : 0;
                if (spheres && rc->n_spheres < max_spheres) spheres[rc->n_spheres] = sp;
                ++rc->n_spheres;
            }
        }
    }

    // checks (what the reference's compile would reject, and what this
    // library does not do)
    if (c.nx < 1 || c.ny < 1 || nz_gpu < 1) r.fail("NX/NY/NZ", "lattice sizes must be >= 1");
    if (rc->steps < 0 || rc->macr_save < 0 || rc->data_report < 0 || rc->ini_step < 0 || rc->checkpoint_save < 0)
        r.fail("steps", "step counts and intervals must be >= 0");
    if (rc->n_gpus != 1)
        throw ParseError{"n_gpus: only 1 is supported (the z-slab decomposition over several GPUs is not built; "
                         "run independent simulations per GPU)", true};
    if (rc->precision_double)
        throw ParseError{"precision: 'double' is not supported: the fused step computes in FP32 on populations "
                         "stored as deviations from the lattice weights (set precision: single)", true};
    if (rc->use_ibm && rc->n_spheres == 0)
        throw ParseError{"use_ibm: true needs at least one sphere under ibm.spheres"};
}

}  // namespace

extern "C" {

vlbm_status vlbm_run_config_parse(const char* yaml_text, vlbm_run_config* out, vlbm_sphere* spheres,
                                  int32_t max_spheres) {
    if (!yaml_text || !out) {
        vlbm::set_last_error("null argument");
        return VLBM_ERR_INVALID;
    }
    vlbm_run_config rc;
    std::memset(&rc, 0, sizeof(rc));
    vlbm_config_default(&rc.cfg);
    vlbm_ibm_config_default(&rc.ibm);
    try {
        Node root = parse_yaml(yaml_text);
        fill(root, &rc, spheres, max_spheres < 0 ? 0 : max_spheres);
    } catch (const ParseError& e) {
        vlbm::set_last_error("configuration: " + e.msg);
        return e.unsupported ? VLBM_ERR_UNSUPPORTED : VLBM_ERR_INVALID;
    }
    *out = rc;
    return VLBM_OK;
}

vlbm_status vlbm_run_config_load(const char* path, vlbm_run_config* out, vlbm_sphere* spheres, int32_t max_spheres) {
    if (!path) {
        vlbm::set_last_error("null path");
        return VLBM_ERR_INVALID;
    }
    FILE* f = std::fopen(path, "rb");
    if (!f) {
        vlbm::set_last_error(std::string("cannot open ") + path);
        return VLBM_ERR_NOT_FOUND;
    }
    std::string text;
    char buf[4096];
    size_t k;
    while ((k = std::fread(buf, 1, sizeof(buf), f)) > 0) text.append(buf, k);
    std::fclose(f);
    return vlbm_run_config_parse(text.c_str(), out, spheres, max_spheres);
}

}  // extern "C"
