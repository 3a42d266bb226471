// qasm.cpp -- OpenQASM 2.0 reader: source text to a qgpu_circuit with the
// steps Quantum++'s reader builds (include/qpp/qasm/qasm.hpp:500-770):
//
//   qreg / creg          registers laid out in declaration order
//   U(t, p, l) q         one 1-qubit gate step per qubit (Qiskit's U matrix,
//                        qasm.hpp:567-586 without QASMTOOLS_QASM2_SPECS)
//   CX a, b              a 2-qubit CNOT gate step per pair (qasm.hpp:592-620)
//   known gates          one joint gate step with qpp's matrix (the
//                        known_matrices table, qasm.hpp:55-200): cx id x y z
//                        h s sdg t tdg rx ry rz cz cy swap ch ccx crz
//   u3 / u2 / u1 / u0 / r  one U step each (their qelib1 bodies are one U)
//   cu1 cu3 cswap        their qelib1 bodies, one step per U or known gate, as
//                        qpp expands them (noise is drawn before each step)
//   crx cry sx sxdg rxx rzz p cp u cu
//                        (not in qpp's qelib1; accepted here as extensions)
//                        one joint gate step with the gate's matrix
//   gate definitions     expanded at every call with the arguments bound
//   measure q -> c       non-destructive single-qubit measurements
//   reset q              one reset step over the arguments
//   barrier              ignored
//   if (c == n) qop      a runtime conditional around the operation's steps
//
// Broadcasting follows the language: whole registers of equal size map
// element by element, single qubits repeat. The parser is written from the
// OpenQASM 2.0 grammar (Cross et al., arXiv:1707.03429).
#include <cmath>
#include <complex>
#include <cstdio>
#include <fstream>
#include <functional>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "capi_common.hpp"
#include "circuit.hpp"

namespace {

using C = std::complex<double>;
using Mat = std::vector<C>; // column-major

const char* kRead = "qpp::qasm::read()";

struct Tok {
    enum Kind { Id, Real, Int, Str, Sym, End } kind = End;
    std::string s;
    double v = 0;
    int line = 0, col = 0;
};

[[noreturn]] void fail(const Tok& t, const std::string& msg) {
    qgpu::raise(QGPU_ERR_INVALID_ARGUMENT, kRead,
                "line " + std::to_string(t.line) + ", column " + std::to_string(t.col) + ": " +
                    msg);
}

std::vector<Tok> lex(const std::string& src) {
    std::vector<Tok> out;
    int line = 1, col = 1;
    size_t i = 0;
    auto adv = [&](size_t k) {
        for (size_t j = 0; j < k; ++j) {
            if (src[i] == '\n') {
                ++line;
                col = 1;
            } else {
                ++col;
            }
            ++i;
        }
    };
    while (i < src.size()) {
        const char ch = src[i];
        if (std::isspace(static_cast<unsigned char>(ch))) {
            adv(1);
            continue;
        }
        if (ch == '/' && i + 1 < src.size() && src[i + 1] == '/') {
            while (i < src.size() && src[i] != '\n') adv(1);
            continue;
        }
        Tok t;
        t.line = line;
        t.col = col;
        if (std::isalpha(static_cast<unsigned char>(ch)) || ch == '_') {
            size_t j = i;
            while (j < src.size() &&
                   (std::isalnum(static_cast<unsigned char>(src[j])) || src[j] == '_'))
                ++j;
            t.kind = Tok::Id;
            t.s = src.substr(i, j - i);
            adv(j - i);
        } else if (std::isdigit(static_cast<unsigned char>(ch)) ||
                   (ch == '.' && i + 1 < src.size() &&
                    std::isdigit(static_cast<unsigned char>(src[i + 1])))) {
            size_t j = i;
            bool real = false;
            while (j < src.size() && std::isdigit(static_cast<unsigned char>(src[j]))) ++j;
            if (j < src.size() && src[j] == '.') {
                real = true;
                ++j;
                while (j < src.size() && std::isdigit(static_cast<unsigned char>(src[j]))) ++j;
            }
            if (j < src.size() && (src[j] == 'e' || src[j] == 'E')) {
                size_t k = j + 1;
                if (k < src.size() && (src[k] == '+' || src[k] == '-')) ++k;
                if (k < src.size() && std::isdigit(static_cast<unsigned char>(src[k]))) {
                    real = true;
                    j = k;
                    while (j < src.size() && std::isdigit(static_cast<unsigned char>(src[j]))) ++j;
                }
            }
            t.kind = real ? Tok::Real : Tok::Int;
            t.s = src.substr(i, j - i);
            t.v = std::stod(t.s);
            adv(j - i);
        } else if (ch == '"') {
            size_t j = i + 1;
            while (j < src.size() && src[j] != '"') ++j;
            if (j >= src.size()) fail(t, "unterminated string");
            t.kind = Tok::Str;
            t.s = src.substr(i + 1, j - i - 1);
            adv(j + 1 - i);
        } else {
            t.kind = Tok::Sym;
            if ((ch == '-' && i + 1 < src.size() && src[i + 1] == '>') ||
                (ch == '=' && i + 1 < src.size() && src[i + 1] == '=')) {
                t.s = src.substr(i, 2);
                adv(2);
            } else {
                t.s = std::string(1, ch);
                adv(1);
            }
        }
        out.push_back(t);
    }
    Tok e;
    e.kind = Tok::End;
    e.line = line;
    e.col = col;
    out.push_back(e);
    return out;
}

// ------------------------------------------------------------- matrices
Mat mat2(C a, C b, C c, C d) { return {a, c, b, d}; } // rows (a b; c d)
Mat ident(int D) {
    Mat m(size_t(D) * D, 0.0);
    for (int i = 0; i < D; ++i) m[i + i * D] = 1.0;
    return m;
}
Mat controlled(const Mat& U) { // |0><0| x I + |1><1| x U (4 x 4)
    Mat m = ident(4);
    for (int r = 0; r < 2; ++r)
        for (int c = 0; c < 2; ++c) m[(2 + r) + 4 * (2 + c)] = U[r + 2 * c];
    return m;
}
const C I1(0.0, 1.0);
Mat gU(double t, double p, double l) {
    return mat2(std::cos(t / 2), -std::exp(I1 * l) * std::sin(t / 2), std::exp(I1 * p) * std::sin(t / 2),
                std::exp(I1 * (p + l)) * std::cos(t / 2));
}
// Rn(theta, axis) = cos(theta/2) I - i sin(theta/2) sigma (gates.hpp:136-143)
Mat gRX(double t) { return mat2(std::cos(t / 2), -I1 * std::sin(t / 2), -I1 * std::sin(t / 2), std::cos(t / 2)); }
Mat gRY(double t) { return mat2(std::cos(t / 2), -std::sin(t / 2), std::sin(t / 2), std::cos(t / 2)); }
Mat gRZ(double t) { return mat2(std::exp(-I1 * (t / 2)), 0.0, 0.0, std::exp(I1 * (t / 2))); }

struct Builtin {
    int nparams, nqubits;
    bool as_u;          // emitted as a U step (u3 / u2 / u1 / u0)
    std::function<Mat(const std::vector<double>&)> m;
};

const std::map<std::string, Builtin>& builtins() {
    static const std::map<std::string, Builtin> b = [] {
        const double r2 = 1 / std::sqrt(2.0);
        const Mat X = mat2(0.0, 1.0, 1.0, 0.0), Y = mat2(0.0, -I1, I1, 0.0), Z = mat2(1.0, 0.0, 0.0, -1.0);
        const Mat H = mat2(r2, r2, r2, -r2), S = mat2(1.0, 0.0, 0.0, I1);
        const Mat T = mat2(1.0, 0.0, 0.0, std::exp(I1 * (M_PI / 4)));
        auto adj = [](const Mat& m) { return mat2(std::conj(m[0]), std::conj(m[1]), std::conj(m[2]), std::conj(m[3])); };
        Mat swap = ident(4);
        swap[1 + 4 * 1] = swap[2 + 4 * 2] = 0.0;
        swap[2 + 4 * 1] = swap[1 + 4 * 2] = 1.0;
        Mat tof = ident(8);
        tof[6 + 8 * 6] = tof[7 + 8 * 7] = 0.0;
        tof[7 + 8 * 6] = tof[6 + 8 * 7] = 1.0;
        Mat cz = ident(4);
        cz[3 + 4 * 3] = -1.0;
        const Mat SX = mat2(C(0.5, 0.5), C(0.5, -0.5), C(0.5, -0.5), C(0.5, 0.5));
        std::map<std::string, Builtin> m;
        auto fixed = [&](const std::string& n, int q, Mat M) {
            m[n] = {0, q, false, [M](const std::vector<double>&) { return M; }};
        };
        fixed("cx", 2, controlled(X));
        fixed("id", 1, ident(2));
        fixed("x", 1, X);
        fixed("y", 1, Y);
        fixed("z", 1, Z);
        fixed("h", 1, H);
        fixed("s", 1, S);
        fixed("sdg", 1, adj(S));
        fixed("t", 1, T);
        fixed("tdg", 1, adj(T));
        fixed("cz", 2, cz);
        fixed("cy", 2, controlled(Y));
        fixed("swap", 2, swap);
        fixed("ch", 2, controlled(H));
        fixed("ccx", 3, tof);
        fixed("sx", 1, SX);
        fixed("sxdg", 1, adj(SX));
        m["rx"] = {1, 1, false, [](const std::vector<double>& a) { return gRX(a[0]); }};
        m["ry"] = {1, 1, false, [](const std::vector<double>& a) { return gRY(a[0]); }};
        m["rz"] = {1, 1, false, [](const std::vector<double>& a) { return gRZ(a[0]); }};
        m["crz"] = {1, 2, false, [](const std::vector<double>& a) { return controlled(gRZ(a[0])); }};
        m["crx"] = {1, 2, false, [](const std::vector<double>& a) { return controlled(gRX(a[0])); }};
        m["cry"] = {1, 2, false, [](const std::vector<double>& a) { return controlled(gRY(a[0])); }};
        m["u3"] = {3, 1, true, [](const std::vector<double>& a) { return gU(a[0], a[1], a[2]); }};
        m["u"] = {3, 1, true, [](const std::vector<double>& a) { return gU(a[0], a[1], a[2]); }};
        m["u2"] = {2, 1, true, [](const std::vector<double>& a) { return gU(M_PI / 2, a[0], a[1]); }};
        m["u1"] = {1, 1, true, [](const std::vector<double>& a) { return gU(0, 0, a[0]); }};
        m["p"] = {1, 1, true, [](const std::vector<double>& a) { return gU(0, 0, a[0]); }};
        m["u0"] = {1, 1, true, [](const std::vector<double>&) { return gU(0, 0, 0); }};
        m["cp"] = {1, 2, false, [](const std::vector<double>& a) { return controlled(gU(0, 0, a[0])); }};
        m["cu"] = {4, 2, false, [](const std::vector<double>& a) {
                       Mat u = gU(a[0], a[1], a[2]);
                       for (C& z : u) z *= std::exp(I1 * a[3]);
                       return controlled(u);
                   }};
        m["rzz"] = {1, 2, false, [](const std::vector<double>& a) {
                        Mat r(16, 0.0);
                        const C e0 = std::exp(-I1 * (a[0] / 2)), e1 = std::exp(I1 * (a[0] / 2));
                        r[0] = e0;
                        r[5] = e1;
                        r[10] = e1;
                        r[15] = e0;
                        return r;
                    }};
        m["rxx"] = {1, 2, false, [](const std::vector<double>& a) {
                        Mat r(16, 0.0);
                        const double c = std::cos(a[0] / 2), s = std::sin(a[0] / 2);
                        for (int i = 0; i < 4; ++i) {
                            r[i + 4 * i] = c;
                            r[(3 - i) + 4 * i] = -I1 * s;
                        }
                        return r;
                    }};
        return m;
    }();
    return b;
}

// ---------------------------------------------------------------- parser
struct GateDef {
    std::vector<std::string> params, args;
    size_t body_begin = 0, body_end = 0; // token range of the body
};

struct Op {
    enum Kind { Gate, Measure, Reset, CondIf, CondEnd } kind = Gate;
    Mat U;
    std::vector<uint64_t> q;
    uint64_t c = 0;
    std::vector<uint64_t> dits;
    uint64_t value = 0;
};

struct Parser {
    std::vector<Tok> t;
    size_t p = 0;
    std::map<std::string, std::pair<uint64_t, uint64_t>> qregs, cregs; // name -> (start, size)
    uint64_t nq = 0, nc = 0;
    std::map<std::string, GateDef> gates;
    std::vector<Op> ops;

    const Tok& peek() const { return t[p]; }
    const Tok& next() { return t[p < t.size() - 1 ? p++ : p]; }
    bool is(const char* s) const { return peek().kind == Tok::Sym && peek().s == s; }
    bool is_id(const char* s) const { return peek().kind == Tok::Id && peek().s == s; }
    void expect(const char* s) {
        if (!is(s)) fail(peek(), std::string("expected '") + s + "'");
        next();
    }
    std::string ident() {
        if (peek().kind != Tok::Id) fail(peek(), "expected an identifier");
        return next().s;
    }
    uint64_t integer() {
        if (peek().kind != Tok::Int) fail(peek(), "expected an integer");
        return uint64_t(next().v);
    }

    // expressions: + - * / ^, unary minus, pi, parameters, functions
    double expr(const std::map<std::string, double>& env) {
        double v = term(env);
        while (is("+") || is("-")) {
            const bool plus = next().s == "+";
            const double r = term(env);
            v = plus ? v + r : v - r;
        }
        return v;
    }
    double term(const std::map<std::string, double>& env) {
        double v = power(env);
        while (is("*") || is("/")) {
            const bool mul = next().s == "*";
            const double r = power(env);
            v = mul ? v * r : v / r;
        }
        return v;
    }
    double power(const std::map<std::string, double>& env) {
        const double b = unary(env);
        if (is("^")) {
            next();
            return std::pow(b, power(env));
        }
        return b;
    }
    double unary(const std::map<std::string, double>& env) {
        if (is("-")) {
            next();
            return -unary(env);
        }
        if (is("+")) {
            next();
            return unary(env);
        }
        return primary(env);
    }
    double primary(const std::map<std::string, double>& env) {
        const Tok& k = peek();
        if (k.kind == Tok::Real || k.kind == Tok::Int) return next().v;
        if (is("(")) {
            next();
            const double v = expr(env);
            expect(")");
            return v;
        }
        if (k.kind == Tok::Id) {
            const std::string n = next().s;
            if (n == "pi") return M_PI;
            static const std::map<std::string, double (*)(double)> fn = {
                {"sin", [](double x) { return std::sin(x); }}, {"cos", [](double x) { return std::cos(x); }},
                {"tan", [](double x) { return std::tan(x); }}, {"exp", [](double x) { return std::exp(x); }},
                {"ln", [](double x) { return std::log(x); }},  {"sqrt", [](double x) { return std::sqrt(x); }}};
            auto f = fn.find(n);
            if (f != fn.end()) {
                expect("(");
                const double v = expr(env);
                expect(")");
                return f->second(v);
            }
            auto e = env.find(n);
            if (e == env.end()) fail(k, "unknown parameter '" + n + "'");
            return e->second;
        }
        fail(k, "expected an expression");
    }

    // a qubit / bit argument: the indices it names
    std::vector<uint64_t> arg(bool quantum, const std::map<std::string, uint64_t>* local) {
        const Tok& k = peek();
        const std::string n = ident();
        if (local) {
            auto it = local->find(n);
            if (it == local->end()) fail(k, "unknown gate argument '" + n + "'");
            return {it->second};
        }
        auto& regs = quantum ? qregs : cregs;
        auto it = regs.find(n);
        if (it == regs.end()) fail(k, std::string("unknown ") + (quantum ? "qreg" : "creg") + " '" + n + "'");
        if (is("[")) {
            next();
            const Tok& ik = peek();
            const uint64_t i = integer();
            expect("]");
            if (i >= it->second.second) fail(ik, "index out of range");
            return {it->second.first + i};
        }
        std::vector<uint64_t> all(it->second.second);
        for (uint64_t i = 0; i < all.size(); ++i) all[i] = it->second.first + i;
        return all;
    }

    void emit_gate(const Mat& U, std::vector<uint64_t> q) {
        Op o;
        o.kind = Op::Gate;
        o.U = U;
        o.q = std::move(q);
        ops.push_back(std::move(o));
    }

    // a gate application (U, CX, a built-in or a defined gate) with its
    // arguments; inside a definition `local` binds argument names
    void qop_gate(const std::map<std::string, double>& env,
                  const std::map<std::string, uint64_t>* local) {
        const Tok& k = peek();
        const std::string name = ident();
        std::vector<double> params;
        if (is("(")) {
            next();
            if (!is(")")) {
                params.push_back(expr(env));
                while (is(",")) {
                    next();
                    params.push_back(expr(env));
                }
            }
            expect(")");
        }
        std::vector<std::vector<uint64_t>> args;
        args.push_back(arg(true, local));
        while (is(",")) {
            next();
            args.push_back(arg(true, local));
        }
        expect(";");
        size_t width = 1;
        for (auto& a : args)
            if (a.size() > 1) {
                if (width > 1 && a.size() != width) fail(k, "registers of different sizes");
                width = a.size();
            }
        auto at = [&](size_t i, size_t j) { return args[i].size() > 1 ? args[i][j] : args[i][0]; };
        if (name == "U") {
            if (params.size() != 3 || args.size() != 1) fail(k, "U takes 3 parameters and 1 argument");
            const Mat u = gU(params[0], params[1], params[2]);
            for (size_t j = 0; j < width; ++j) emit_gate(u, {at(0, j)});
            return;
        }
        if (name == "CX") {
            if (!params.empty() || args.size() != 2) fail(k, "CX takes 2 arguments");
            const Mat cx = builtins().at("cx").m({});
            for (size_t j = 0; j < width; ++j) emit_gate(cx, {at(0, j), at(1, j)});
            return;
        }
        auto d = gates.find(name);
        if (d != gates.end()) { // a definition of the file: expand its body
            const GateDef& g = d->second;
            if (params.size() != g.params.size() || args.size() != g.args.size())
                fail(k, "wrong number of parameters or arguments for '" + name + "'");
            for (size_t j = 0; j < width; ++j) {
                std::map<std::string, double> env2;
                for (size_t i = 0; i < params.size(); ++i) env2[g.params[i]] = params[i];
                std::map<std::string, uint64_t> loc;
                for (size_t i = 0; i < args.size(); ++i) loc[g.args[i]] = at(i, j);
                const size_t save = p;
                p = g.body_begin;
                while (p < g.body_end) body_stmt(env2, &loc);
                p = save;
            }
            return;
        }
        // qelib1 gates that Quantum++'s reader expands into their bodies
        // (the standard library text of qasmtools/include/qasmtools/parser/
        // preprocessor.hpp:86-127, used when QASMTOOLS_QASM2_SPECS is not
        // defined): one step per U / known gate of the body, so a noisy
        // engine draws noise before each of them as qpp does
        if (name == "cu1" || name == "cu3" || name == "cswap" || name == "r") {
            const size_t np = name == "cu1" ? 1 : name == "cu3" ? 3 : name == "r" ? 2 : 0;
            const size_t nq = name == "cswap" ? 3 : name == "r" ? 1 : 2;
            if (params.size() != np || args.size() != nq)
                fail(k, "wrong number of parameters or arguments for '" + name + "'");
            const Mat cx = builtins().at("cx").m({});
            for (size_t j = 0; j < width; ++j) {
                const uint64_t a = at(0, j);
                if (name == "r") { // u3(theta, phi - pi/2, -phi + pi/2)
                    emit_gate(gU(params[0], params[1] - M_PI / 2, -params[1] + M_PI / 2), {a});
                } else if (name == "cu1") {
                    const uint64_t b2 = at(1, j);
                    const double l = params[0];
                    emit_gate(gU(0, 0, l / 2), {a});
                    emit_gate(cx, {a, b2});
                    emit_gate(gU(0, 0, -l / 2), {b2});
                    emit_gate(cx, {a, b2});
                    emit_gate(gU(0, 0, l / 2), {b2});
                } else if (name == "cu3") {
                    const uint64_t t = at(1, j);
                    const double th = params[0], ph = params[1], l = params[2];
                    emit_gate(gU(0, 0, (l + ph) / 2), {a});
                    emit_gate(gU(0, 0, (l - ph) / 2), {t});
                    emit_gate(cx, {a, t});
                    emit_gate(gU(-th / 2, 0, -(ph + l) / 2), {t});
                    emit_gate(cx, {a, t});
                    emit_gate(gU(th / 2, ph, 0), {t});
                } else { // cswap a, b, c: cx c,b; ccx a,b,c; cx c,b
                    const uint64_t b2 = at(1, j), c2 = at(2, j);
                    emit_gate(cx, {c2, b2});
                    emit_gate(builtins().at("ccx").m({}), {a, b2, c2});
                    emit_gate(cx, {c2, b2});
                }
            }
            return;
        }
        auto b = builtins().find(name);
        if (b == builtins().end()) fail(k, "unknown gate '" + name + "'");
        if (int(params.size()) != b->second.nparams || int(args.size()) != b->second.nqubits)
            fail(k, "wrong number of parameters or arguments for '" + name + "'");
        const Mat M = b->second.m(params);
        for (size_t j = 0; j < width; ++j) {
            std::vector<uint64_t> q;
            for (size_t i = 0; i < args.size(); ++i) q.push_back(at(i, j));
            emit_gate(M, q);
        }
    }

    void body_stmt(const std::map<std::string, double>& env,
                   const std::map<std::string, uint64_t>* local) {
        if (is_id("barrier")) {
            while (!is(";")) next();
            next();
            return;
        }
        qop_gate(env, local);
    }

    // measure / reset / gate (the operation of a statement or an if)
    void qop() {
        static const std::map<std::string, double> none;
        if (is_id("measure")) {
            const Tok& k = next();
            std::vector<uint64_t> q = arg(true, nullptr);
            expect("->");
            std::vector<uint64_t> c = arg(false, nullptr);
            expect(";");
            if (q.size() != c.size()) fail(k, "measure: sizes differ");
            for (size_t i = 0; i < q.size(); ++i) {
                Op o;
                o.kind = Op::Measure;
                o.q = {q[i]};
                o.c = c[i];
                ops.push_back(o);
            }
            return;
        }
        if (is_id("reset")) {
            next();
            Op o;
            o.kind = Op::Reset;
            o.q = arg(true, nullptr);
            expect(";");
            ops.push_back(o);
            return;
        }
        qop_gate(none, nullptr);
    }

    void statement() {
        const Tok& k = peek();
        if (is_id("include")) {
            next();
            if (peek().kind != Tok::Str) fail(peek(), "expected a file name");
            const std::string f = next().s;
            expect(";");
            if (f != "qelib1.inc") fail(k, "only qelib1.inc can be included");
            return;
        }
        if (is_id("qreg") || is_id("creg")) {
            const bool q = next().s == "qreg";
            const std::string n = ident();
            expect("[");
            const uint64_t sz = integer();
            expect("]");
            expect(";");
            auto& regs = q ? qregs : cregs;
            if (regs.count(n)) fail(k, "register '" + n + "' declared twice");
            uint64_t& tot = q ? nq : nc;
            regs[n] = {tot, sz};
            tot += sz;
            return;
        }
        if (is_id("gate")) {
            next();
            const std::string n = ident();
            GateDef g;
            if (is("(")) {
                next();
                if (!is(")")) {
                    g.params.push_back(ident());
                    while (is(",")) {
                        next();
                        g.params.push_back(ident());
                    }
                }
                expect(")");
            }
            g.args.push_back(ident());
            while (is(",")) {
                next();
                g.args.push_back(ident());
            }
            expect("{");
            g.body_begin = p;
            int depth = 1;
            while (depth > 0) {
                if (peek().kind == Tok::End) fail(peek(), "unterminated gate body");
                if (is("{")) ++depth;
                if (is("}")) --depth;
                if (depth > 0) next();
            }
            g.body_end = p;
            next(); // '}'
            gates[n] = g;
            return;
        }
        if (is_id("opaque")) fail(k, "opaque gates are not supported");
        if (is_id("barrier")) {
            while (!is(";")) next();
            next();
            return;
        }
        if (is_id("if")) {
            next();
            expect("(");
            const Tok& rk = peek();
            const std::string r = ident();
            expect("==");
            const uint64_t v = integer();
            expect(")");
            auto it = cregs.find(r);
            if (it == cregs.end()) fail(rk, "unknown creg '" + r + "'");
            Op o;
            o.kind = Op::CondIf;
            for (uint64_t i = 0; i < it->second.second; ++i) o.dits.push_back(it->second.first + i);
            o.value = v;
            ops.push_back(o);
            qop();
            Op e;
            e.kind = Op::CondEnd;
            ops.push_back(e);
            return;
        }
        qop();
    }

    void program() {
        if (!is_id("OPENQASM")) fail(peek(), "expected 'OPENQASM 2.0;'");
        next();
        const Tok& v = peek();
        if (v.kind != Tok::Real || v.v != 2.0) fail(v, "only OpenQASM 2.0 is supported");
        next();
        expect(";");
        while (peek().kind != Tok::End) statement();
    }
};

qgpu_circuit* build(const std::string& src) {
    Parser P;
    P.t = lex(src);
    P.program();
    if (P.nq == 0) qgpu::raise(QGPU_ERR_ZERO_SIZE, kRead, "no qubits declared");
    qgpu_circuit* c = nullptr;
    auto ok = [&](qgpu_status s) {
        if (s != QGPU_OK) qgpu::raise(s, qgpu_last_error_where(), qgpu_last_error_what());
    };
    ok(qgpu_circuit_create(uint32_t(P.nq), 2, uint32_t(P.nc), &c));
    try {
        for (const Op& o : P.ops) {
            switch (o.kind) {
                case Op::Gate:
                    ok(qgpu_circuit_gate(c, reinterpret_cast<const double*>(o.U.data()),
                                         uint64_t(1) << o.q.size(), o.q.data(), uint32_t(o.q.size())));
                    break;
                case Op::Measure:
                    ok(qgpu_circuit_measure(c, o.q.data(), 1, o.c, 0));
                    break;
                case Op::Reset:
                    ok(qgpu_circuit_reset(c, o.q.data(), uint32_t(o.q.size())));
                    break;
                case Op::CondIf:
                    ok(qgpu_circuit_cond_if(c, o.dits.data(), uint32_t(o.dits.size()), o.value));
                    break;
                case Op::CondEnd:
                    ok(qgpu_circuit_cond_end(c));
                    break;
            }
        }
    } catch (...) {
        qgpu_circuit_destroy(c);
        throw;
    }
    return c;
}

} // namespace

extern "C" {

// qpp::qasm::read_from_string (qasm.hpp:800-806)
qgpu_status qgpu_qasm_read(const char* source, qgpu_circuit** out) {
    return qgpu::guarded(__func__, [&] {
        if (!source || !out) qgpu::raise(QGPU_ERR_INVALID_ARGUMENT, kRead, "source/out");
        *out = build(source);
    });
}

// qpp::qasm::read_from_file (qasm.hpp:815-820)
qgpu_status qgpu_qasm_read_file(const char* path, qgpu_circuit** out) {
    return qgpu::guarded(__func__, [&] {
        if (!path || !out) qgpu::raise(QGPU_ERR_INVALID_ARGUMENT, kRead, "path/out");
        std::ifstream f(path);
        if (!f) qgpu::raise(QGPU_ERR_INVALID_ARGUMENT, kRead, std::string("cannot open ") + path);
        std::stringstream ss;
        ss << f.rdbuf();
        *out = build(ss.str());
    });
}

} // extern "C"
