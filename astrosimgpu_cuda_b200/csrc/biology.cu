// biology.cu -- the biology parameter table and the JSON override loader.

#include <cctype>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <set>
#include <string>

#include "biology.cuh"

namespace astrosim {

namespace {

enum class Kind { Real, Flag, Int };

struct Field {
    const char* name;
    Kind kind;
    size_t offset;
};

#define AS_REAL(f) {#f, Kind::Real, offsetof(Biology, f)},
#define AS_FLAG(f) {#f, Kind::Flag, offsetof(Biology, f)},
#define AS_INT(f) {#f, Kind::Int, offsetof(Biology, f)},

// Every field of Biology, in declaration order.
const Field kFields[] = {
    AS_REAL(Ca_tot) AS_REAL(IP3_0) AS_REAL(tau_IP3) AS_REAL(delta_IP3) AS_REAL(SIC_scale) AS_REAL(Kd_IP3_1)
    AS_REAL(Kd_IP3_2) AS_REAL(Kd_act) AS_REAL(Kd_inh) AS_REAL(Km_SERCA) AS_REAL(SIC_th) AS_REAL(k_IP3R)
    AS_REAL(rate_IP3R) AS_REAL(rate_L) AS_REAL(rate_SERCA) AS_REAL(ratio_ER_cyt) AS_REAL(Ca_init) AS_REAL(h_init)
    AS_REAL(IP3_init) AS_FLAG(randomize_astro) AS_REAL(ra_lower) AS_REAL(ra_upper) AS_REAL(ra_var)
    AS_REAL(e_Delta_T) AS_REAL(e_a) AS_REAL(e_tau_w) AS_REAL(e_V_reset) AS_REAL(e_b) AS_REAL(e_V_m) AS_REAL(e_C_m)
    AS_REAL(e_g_L) AS_REAL(e_E_L) AS_REAL(e_V_th) AS_REAL(e_V_peak) AS_REAL(e_t_ref) AS_REAL(e_E_ex)
    AS_REAL(e_E_in) AS_REAL(e_tau_syn_ex) AS_REAL(e_tau_syn_in)
    AS_REAL(i_Delta_T) AS_REAL(i_a) AS_REAL(i_tau_w) AS_REAL(i_V_reset) AS_REAL(i_b) AS_REAL(i_V_m) AS_REAL(i_C_m)
    AS_REAL(i_g_L) AS_REAL(i_E_L) AS_REAL(i_V_th) AS_REAL(i_V_peak) AS_REAL(i_t_ref) AS_REAL(i_E_ex)
    AS_REAL(i_E_in) AS_REAL(i_tau_syn_ex) AS_REAL(i_tau_syn_in)
    AS_FLAG(randomize_neuron) AS_REAL(rn_lower) AS_REAL(rn_upper) AS_REAL(rn_var)
    AS_REAL(w_e) AS_REAL(w_i) AS_REAL(w_n2a) AS_REAL(w_a2n) AS_REAL(d_e) AS_REAL(d_i) AS_REAL(d_a2n)
    AS_FLAG(stp_enabled) AS_REAL(stp_U) AS_REAL(stp_tau_rec) AS_REAL(stp_tau_fac) AS_INT(sic_interval)
    AS_REAL(astro_poiss_rate) AS_REAL(astro_poiss_weight) AS_REAL(astro_noise_std)
    AS_REAL(exc_poiss_rate) AS_REAL(exc_poiss_weight) AS_REAL(exc_noise_std)
    AS_REAL(inh_poiss_rate) AS_REAL(inh_poiss_weight) AS_REAL(inh_noise_std)
    AS_FLAG(independent_noise) AS_REAL(noise_dt)
};

#undef AS_REAL
#undef AS_FLAG
#undef AS_INT

const Field* find_field(const std::string& name) {
    for (const Field& f : kFields)
        if (name == f.name) return &f;
    return nullptr;
}

// A minimal reader for one flat JSON object of string keys and number / boolean values.
struct Reader {
    const char* p;
    void ws() {
        while (*p && std::isspace(static_cast<unsigned char>(*p))) ++p;
    }
    bool eat(char c) {
        ws();
        if (*p != c) return false;
        ++p;
        return true;
    }
    bool string(std::string& out) {
        ws();
        if (*p != '"') return false;
        ++p;
        out.clear();
        while (*p && *p != '"') {
            if (*p == '\\') return false;  // parameter names need no escapes
            out.push_back(*p++);
        }
        if (*p != '"') return false;
        ++p;
        return true;
    }
    // number, true or false; *is_bool tells which
    bool value(double& v, bool& is_bool) {
        ws();
        if (std::strncmp(p, "true", 4) == 0) { p += 4; v = 1.0; is_bool = true; return true; }
        if (std::strncmp(p, "false", 5) == 0) { p += 5; v = 0.0; is_bool = true; return true; }
        if (!(*p == '-' || std::isdigit(static_cast<unsigned char>(*p)))) return false;
        char* end = nullptr;
        v = std::strtod(p, &end);
        if (end == p) return false;
        p = end;
        is_bool = false;
        return true;
    }
};

Status set_field(Biology& bio, const Field& f, double v, bool is_bool) {
    char* base = reinterpret_cast<char*>(&bio) + f.offset;
    switch (f.kind) {
        case Kind::Real:
            if (is_bool) return make_error(ASTROSIM_ERR_INVALID_ARG, "biology parameter '%s' takes a number", f.name);
            if (!std::isfinite(v)) return make_error(ASTROSIM_ERR_INVALID_ARG, "biology parameter '%s' is not finite", f.name);
            *reinterpret_cast<double*>(base) = v;
            return Status::Ok();
        case Kind::Flag:
            if (v != 0.0 && v != 1.0)
                return make_error(ASTROSIM_ERR_INVALID_ARG, "biology parameter '%s' takes true or false", f.name);
            *reinterpret_cast<bool*>(base) = v != 0.0;
            return Status::Ok();
        case Kind::Int:
            if (is_bool || v != std::floor(v) || std::fabs(v) > 1e9)
                return make_error(ASTROSIM_ERR_INVALID_ARG, "biology parameter '%s' takes an integer", f.name);
            *reinterpret_cast<int*>(base) = static_cast<int>(v);
            return Status::Ok();
    }
    return Status::Ok();
}

// Values the kernels divide by or count with must stay in range.
Status validate(const Biology& b) {
    struct Pos { const char* name; double v; };
    const Pos positive[] = {
        {"tau_IP3", b.tau_IP3}, {"ratio_ER_cyt", b.ratio_ER_cyt}, {"Km_SERCA", b.Km_SERCA},
        {"e_C_m", b.e_C_m}, {"e_tau_w", b.e_tau_w}, {"e_Delta_T", b.e_Delta_T},
        {"e_tau_syn_ex", b.e_tau_syn_ex}, {"e_tau_syn_in", b.e_tau_syn_in},
        {"i_C_m", b.i_C_m}, {"i_tau_w", b.i_tau_w}, {"i_Delta_T", b.i_Delta_T},
        {"i_tau_syn_ex", b.i_tau_syn_ex}, {"i_tau_syn_in", b.i_tau_syn_in},
        {"d_e", b.d_e}, {"d_i", b.d_i}, {"d_a2n", b.d_a2n}, {"stp_tau_rec", b.stp_tau_rec}};
    for (const Pos& q : positive)
        if (!(q.v > 0.0)) return make_error(ASTROSIM_ERR_INVALID_ARG, "biology parameter '%s' must be > 0", q.name);
    const Pos nonneg[] = {
        {"e_t_ref", b.e_t_ref}, {"i_t_ref", b.i_t_ref}, {"ra_var", b.ra_var}, {"rn_var", b.rn_var},
        {"stp_tau_fac", b.stp_tau_fac}, {"astro_poiss_rate", b.astro_poiss_rate},
        {"exc_poiss_rate", b.exc_poiss_rate}, {"inh_poiss_rate", b.inh_poiss_rate},
        {"astro_noise_std", b.astro_noise_std}, {"exc_noise_std", b.exc_noise_std},
        {"inh_noise_std", b.inh_noise_std}, {"noise_dt", b.noise_dt}};
    for (const Pos& q : nonneg)
        if (!(q.v >= 0.0)) return make_error(ASTROSIM_ERR_INVALID_ARG, "biology parameter '%s' must be >= 0", q.name);
    if (b.sic_interval < 1) return make_error(ASTROSIM_ERR_INVALID_ARG, "biology parameter 'sic_interval' must be >= 1");
    if (b.randomize_astro && !(b.ra_lower < b.ra_upper))
        return make_error(ASTROSIM_ERR_INVALID_ARG, "biology parameters need ra_lower < ra_upper");
    if (b.randomize_neuron && !(b.rn_lower < b.rn_upper))
        return make_error(ASTROSIM_ERR_INVALID_ARG, "biology parameters need rn_lower < rn_upper");
    if (!(b.stp_U > 0.0 && b.stp_U <= 1.0))
        return make_error(ASTROSIM_ERR_INVALID_ARG, "biology parameter 'stp_U' must be in (0, 1]");
    return Status::Ok();
}

}  // namespace

Status apply_biology_json(const char* json, Biology& bio) {
    if (!json) return Status::Ok();
    Reader r{json};
    r.ws();
    if (!*r.p) return Status::Ok();
    Biology b = bio;
    if (!r.eat('{')) return make_error(ASTROSIM_ERR_INVALID_ARG, "biology JSON: expected '{'");
    std::set<std::string> seen;
    if (!r.eat('}')) {
        for (;;) {
            std::string key;
            if (!r.string(key)) return make_error(ASTROSIM_ERR_INVALID_ARG, "biology JSON: expected a quoted name");
            if (!r.eat(':')) return make_error(ASTROSIM_ERR_INVALID_ARG, "biology JSON: expected ':' after '%s'", key.c_str());
            double v = 0.0;
            bool is_bool = false;
            if (!r.value(v, is_bool))
                return make_error(ASTROSIM_ERR_INVALID_ARG, "biology JSON: '%s' needs a number, true or false", key.c_str());
            const Field* f = find_field(key);
            if (!f) return make_error(ASTROSIM_ERR_INVALID_ARG, "unknown biology parameter '%s'", key.c_str());
            if (!seen.insert(key).second)
                return make_error(ASTROSIM_ERR_INVALID_ARG, "biology parameter '%s' given twice", key.c_str());
            AS_TRY(set_field(b, *f, v, is_bool));
            if (r.eat(',')) continue;
            if (r.eat('}')) break;
            return make_error(ASTROSIM_ERR_INVALID_ARG, "biology JSON: expected ',' or '}' after '%s'", key.c_str());
        }
    }
    r.ws();
    if (*r.p) return make_error(ASTROSIM_ERR_INVALID_ARG, "biology JSON: text after the closing '}'");
    AS_TRY(validate(b));
    bio = b;
    return Status::Ok();
}

std::string biology_names() {
    std::string s;
    for (const Field& f : kFields) {
        if (!s.empty()) s += ',';
        s += f.name;
    }
    return s;
}

Status biology_get(const Biology& bio, const char* name, double* value) {
    if (!name || !value) return make_error(ASTROSIM_ERR_INVALID_ARG, "null argument");
    const Field* f = find_field(name);
    if (!f) return make_error(ASTROSIM_ERR_INVALID_ARG, "unknown biology parameter '%s'", name);
    const char* base = reinterpret_cast<const char*>(&bio) + f->offset;
    switch (f->kind) {
        case Kind::Real: *value = *reinterpret_cast<const double*>(base); break;
        case Kind::Flag: *value = *reinterpret_cast<const bool*>(base) ? 1.0 : 0.0; break;
        case Kind::Int: *value = *reinterpret_cast<const int*>(base); break;
    }
    return Status::Ok();
}

}  // namespace astrosim
