// cpx-pi -- command-line front end: exact pi(x) on one GPU.
//
// Replaces the reference's CLI (src/main.cpp:23-194), which parsed x by
// running the external `calc` program through popen and chose y with a
// floating-point alpha(x).  Here x is parsed exactly in 128-bit integers from
// an expression (decimal literals, AeB = A * 10^B, A^B, *, +, -, parentheses),
// y follows the library's rule (alpha(x) of src/main.cpp:128-194, or --alpha /
// --y), and the result is printed as text or one JSON line.
//
//   cpx-pi 1e20 --alpha 16 --terms --json
//   cpx-pi --batch xs.txt            (one expression per line; one batched pass)
//   cpx-pi --parse '2^64+13'         (print the parsed x; no GPU needed)
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/cpx.h"

typedef unsigned __int128 u128;
typedef __int128 i128;

namespace {

const u128 kMax = ~(u128)0;

u128 mul_chk(u128 a, u128 b)
{
    if (a && b > kMax / a) throw std::runtime_error("x does not fit in 128 bits");
    return a * b;
}
u128 add_chk(u128 a, u128 b)
{
    if (b > kMax - a) throw std::runtime_error("x does not fit in 128 bits");
    return a + b;
}
u128 pow_chk(u128 a, u128 e)
{
    u128 r = 1;
    for (u128 i = 0; i < e; i++) {
        r = mul_chk(r, a);
        if (i > 200) throw std::runtime_error("exponent too large");
    }
    return r;
}

// recursive descent over: expr = term (('+'|'-') term)*; term = pow ('*' pow)*;
// pow = atom ('^' pow)?; atom = number ['e' number] | '(' expr ')'
struct Parser {
    const char *s;
    size_t i = 0;
    void ws()
    {
        while (s[i] == ' ' || s[i] == '\t') i++;
    }
    u128 number()
    {
        ws();
        if (s[i] < '0' || s[i] > '9') throw std::runtime_error(std::string("expected a number at: ") + (s + i));
        u128 v = 0;
        while (s[i] >= '0' && s[i] <= '9') {
            v = add_chk(mul_chk(v, 10), (u128)(s[i] - '0'));
            i++;
            while (s[i] == '_' || s[i] == ',') i++;
        }
        return v;
    }
    u128 atom()
    {
        ws();
        if (s[i] == '(') {
            i++;
            const u128 v = expr();
            ws();
            if (s[i] != ')') throw std::runtime_error("missing )");
            i++;
            return v;
        }
        u128 v = number();
        if (s[i] == 'e' || s[i] == 'E') {
            i++;
            v = mul_chk(v, pow_chk(10, number()));
        }
        return v;
    }
    u128 power()
    {
        const u128 b = atom();
        ws();
        if (s[i] == '^') {
            i++;
            return pow_chk(b, power());
        }
        return b;
    }
    u128 term()
    {
        u128 v = power();
        for (;;) {
            ws();
            if (s[i] != '*') return v;
            i++;
            v = mul_chk(v, power());
        }
    }
    u128 expr()
    {
        u128 v = term();
        for (;;) {
            ws();
            if (s[i] == '+') {
                i++;
                v = add_chk(v, term());
            } else if (s[i] == '-') {
                i++;
                const u128 t = term();
                if (t > v) throw std::runtime_error("negative x");
                v -= t;
            } else {
                return v;
            }
        }
    }
};

u128 parse_x(const std::string &text)
{
    Parser p{text.c_str()};
    const u128 v = p.expr();
    p.ws();
    if (p.s[p.i]) throw std::runtime_error("unexpected text: " + std::string(p.s + p.i));
    return v;
}

std::string dec(u128 v)
{
    if (!v) return "0";
    std::string r;
    while (v) {
        r.insert(r.begin(), char('0' + (int)(v % 10)));
        v /= 10;
    }
    return r;
}
std::string sdec(cpx_u128 v)
{
    const i128 s = (i128)(((u128)v.hi << 64) | v.lo);
    return s < 0 ? "-" + dec((u128)(-s)) : dec((u128)s);
}
cpx_u128 C(u128 v) { return cpx_u128{(uint64_t)v, (uint64_t)(v >> 64)}; }

void usage()
{
    std::fprintf(stderr,
                 "usage: cpx-pi X [--alpha A] [--y Y] [--c C] [--terms] [--json] [--device D]\n"
                 "       cpx-pi --batch FILE [--alpha A] [--json] [--device D]\n"
                 "       cpx-pi --parse X\n"
                 "X: decimal integer expression with e-notation, ^, *, +, -, parentheses (e.g. 1e20, 2^64+13)\n");
}

int fail_ctx(cpx_ctx *ctx, int rc, const char *what)
{
    std::fprintf(stderr, "cpx-pi: %s failed (%d): %s\n", what, rc, ctx ? cpx_last_error(ctx) : "");
    return 2;
}

}  // namespace

int main(int argc, char **argv)
{
    std::string xs_arg, batch_file, alpha_s;
    uint64_t y = 0;
    unsigned c = 6;
    int device = 0;
    bool terms = false, json = false, parse_only = false;
    try {
        for (int i = 1; i < argc; i++) {
            const std::string a = argv[i];
            auto next = [&]() -> std::string {
                if (i + 1 >= argc) throw std::runtime_error("missing value after " + a);
                return argv[++i];
            };
            if (a == "--alpha") alpha_s = next();
            else if (a == "--y") y = (uint64_t)parse_x(next());
            else if (a == "--c") c = (unsigned)std::stoul(next());
            else if (a == "--device") device = std::stoi(next());
            else if (a == "--batch") batch_file = next();
            else if (a == "--terms") terms = true;
            else if (a == "--json") json = true;
            else if (a == "--parse") parse_only = true;
            else if (a == "-h" || a == "--help") {
                usage();
                return 0;
            } else if (xs_arg.empty() && a[0] != '-') xs_arg = a;
            else throw std::runtime_error("unknown argument " + a);
        }
        if (parse_only) {
            if (xs_arg.empty()) throw std::runtime_error("--parse needs X");
            std::printf("%s\n", dec(parse_x(xs_arg)).c_str());
            return 0;
        }
        if (xs_arg.empty() == batch_file.empty()) {
            usage();
            return 1;
        }
    } catch (const std::exception &e) {
        std::fprintf(stderr, "cpx-pi: %s\n", e.what());
        return 1;
    }
    // alpha as a fraction num/den (three decimals), 0/0 = the library's alpha(x)
    uint32_t an = 0, ad = 0;
    if (!alpha_s.empty()) {
        const double a = std::atof(alpha_s.c_str());
        if (!(a >= 1.0)) {
            std::fprintf(stderr, "cpx-pi: alpha must be >= 1\n");
            return 1;
        }
        an = (uint32_t)(a * 1000.0 + 0.5);
        ad = 1000;
    }
    cpx_ctx *ctx = nullptr;
    int rc = cpx_create(device, &ctx);
    if (rc) return fail_ctx(nullptr, rc, "cpx_create");
    const auto t0 = std::chrono::steady_clock::now();
    auto ms = [&] { return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count(); };
    if (!batch_file.empty()) {
        std::ifstream f(batch_file);
        if (!f) {
            std::fprintf(stderr, "cpx-pi: cannot read %s\n", batch_file.c_str());
            return 1;
        }
        std::vector<cpx_u128> xv;
        std::string line;
        try {
            while (std::getline(f, line)) {
                const size_t h = line.find('#');
                if (h != std::string::npos) line.resize(h);
                if (line.find_first_not_of(" \t\r") == std::string::npos) continue;
                while (!line.empty() && (line.back() == '\r' || line.back() == ' ')) line.pop_back();
                xv.push_back(C(parse_x(line)));
            }
        } catch (const std::exception &e) {
            std::fprintf(stderr, "cpx-pi: %s\n", e.what());
            return 1;
        }
        std::vector<cpx_u128> out(xv.size());
        cpx_params prm = {};
        prm.alpha_num = an;
        prm.alpha_den = ad;
        prm.c = (uint16_t)c;
        rc = cpx_pi_batch(ctx, xv.data(), xv.size(), &prm, out.data());
        if (rc) return fail_ctx(ctx, rc, "cpx_pi_batch");
        const double t = ms();
        for (size_t i = 0; i < xv.size(); i++) {
            const std::string xd = dec(((u128)xv[i].hi << 64) | xv[i].lo), pd = dec(((u128)out[i].hi << 64) | out[i].lo);
            if (json) std::printf("{\"x\": \"%s\", \"pi\": \"%s\"}\n", xd.c_str(), pd.c_str());
            else std::printf("%s %s\n", xd.c_str(), pd.c_str());
        }
        std::fprintf(stderr, "cpx-pi: %zu queries in %.3f ms\n", xv.size(), t);
        cpx_destroy(ctx);
        return 0;
    }
    u128 x;
    try {
        x = parse_x(xs_arg);
    } catch (const std::exception &e) {
        std::fprintf(stderr, "cpx-pi: %s\n", e.what());
        return 1;
    }
    if (!y && an) {
        rc = cpx_default_y(C(x), an, ad, &y);
        if (rc) return fail_ctx(ctx, rc, "cpx_default_y");
    }
    cpx_terms T = {};
    cpx_u128 pi = {};
    rc = cpx_pi_u128(ctx, C(x), y, (uint16_t)c, &pi, &T);
    if (rc) return fail_ctx(ctx, rc, "cpx_pi_u128");
    const double t = ms();
    if (json) {
        std::printf("{\"x\": \"%s\", \"pi\": \"%s\", \"y\": %llu, \"z\": %llu, \"c\": %u, \"ms\": %.3f",
                    dec(x).c_str(), sdec(pi).c_str(), (unsigned long long)T.y, (unsigned long long)T.z, c, t);
        if (terms)
            std::printf(", \"terms\": {\"P2\": \"%s\", \"ordinary\": \"%s\", \"trivial\": \"%s\", \"easy\": \"%s\", "
                        "\"hard\": \"%s\", \"pi_y\": \"%s\"}",
                        sdec(T.P2).c_str(), sdec(T.ordinary).c_str(), sdec(T.trivial).c_str(), sdec(T.easy).c_str(),
                        sdec(T.hard).c_str(), sdec(T.pi_y).c_str());
        std::printf("}\n");
    } else {
        std::printf("pi(%s) = %s\n", dec(x).c_str(), sdec(pi).c_str());
        if (terms)
            std::printf("  y = %llu, z = %llu, c = %u\n  P2 = %s\n  ordinary = %s\n  trivial = %s\n  easy = %s\n"
                        "  hard = %s\n  pi(y) = %s\n",
                        (unsigned long long)T.y, (unsigned long long)T.z, c, sdec(T.P2).c_str(),
                        sdec(T.ordinary).c_str(), sdec(T.trivial).c_str(), sdec(T.easy).c_str(),
                        sdec(T.hard).c_str(), sdec(T.pi_y).c_str());
        std::printf("  %.3f ms\n", t);
    }
    cpx_destroy(ctx);
    return 0;
}
