// NAMELIST subset reader for the solver controls deck.
//
// The reference reads one namelist group, /InputVariables/ ivd, whose single
// member is a derived type, so a deck holds "ivd%field = value" items
// (def_par:213, 384; SolverExampleInput/C13_1.inp:1-84).  This reader accepts
// that form: items separated by commas or blanks, '!' comments, logicals as
// .true./.false./T/F, reals with E or D exponents, quoted strings, and the
// array elements datum(i), inflowField(i,j), enginesFrontMassFlow(i) and
// enginesRearParameters(i,j).  Keys are matched without
// regard to case, as Fortran does.  Keys the hot path does not use are listed
// back to the caller and otherwise ignored.
#include <cctype>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "flite_prepro.h"

namespace {

enum Kind { INT, DBL, LOG };
struct Field {
    const char *name;
    Kind kind;
    size_t off;
};

#define F_I(n) {#n, INT, offsetof(flite_controls, n)}
#define F_D(n) {#n, DBL, offsetof(flite_controls, n)}
#define F_L(n) {#n, LOG, offsetof(flite_controls, n)}

const Field kFields[] = {
    F_D(MachNumber), F_D(alpha), F_D(beta), F_D(ReynoldsNumber), F_D(PrandtlNumber),
    F_D(gamma), F_D(inflowTemperature), F_D(wallTemperature), F_L(wallsAreIsentropic),
    F_I(fluxType), F_I(HLLCFluxOrder), F_D(HLLCClipping), F_I(Automaticlipping),
    F_I(GradientMethod), F_I(dissipationScheme), F_I(coarseGridDissipationScheme),
    F_D(secondOrderDissipationFactor), F_D(fourthOrderDissipationFactor),
    F_D(coarseGridDissipationFactor), F_L(useMatrixDissipation), F_D(HartensCorrectionFactor),
    F_L(useDissipationWeighting), F_I(viscosityScheme), F_I(boundaryTerm), F_D(CFLNumber),
    F_D(turbulentCFLNumber), F_D(turbK), F_D(maxIncrementFactor), F_D(minimumDensity),
    F_I(multigridScheme), F_I(numberOfRelaxationSteps), F_I(numberOfGridsToUse),
    F_D(multigridBCRelaxation), F_D(prolongationRelaxation), F_D(turbProlongationRelaxation),
    F_I(prolongationMappingScheme), F_I(numberOfMGIterations), F_I(maximumnumberofcycles),
    F_I(writeToFileInterval), F_D(initialResidual), F_I(numberOfCFLIncrements),
    F_I(turbulenceModel), F_I(numberOfTurbulenceGrids), F_I(numberOfTurbulenceSteps),
    F_D(tripFactor), F_D(triggerRadius), F_D(turbulenceTriggerValue), F_I(numberOfTriggerSteps),
    F_D(maxTurbulenceValue), F_D(turbulentPrandtlNumber), F_D(referenceArea), F_D(groundplane),
    F_I(forceCalcType), F_I(restartNumber), F_I(numberOfProcesses), F_I(flowType),
    {"explicit", LOG, offsetof(flite_controls, explicit_)}, F_L(SAS), F_L(GUSTMODEL),
    F_L(movingwall), F_L(patchInitialization), F_I(nspan), F_I(timeScheme), F_I(numberOfRSSteps),
    F_I(numberOfPSSteps), F_D(residualSmoothingFactor), F_D(prolongationSmoothingFactor),
    F_D(physicalTimeStep), F_D(engineBCRelaxation), F_I(engineFlowType),
    F_I(numberOfEORelaxationSteps),
};

bool ieq(const std::string &a, const char *b) {
    size_t n = std::strlen(b);
    if (a.size() != n) return false;
    for (size_t i = 0; i < n; ++i)
        if (std::tolower((unsigned char)a[i]) != std::tolower((unsigned char)b[i])) return false;
    return true;
}

std::string lower(std::string s) {
    for (auto &c : s) c = (char)std::tolower((unsigned char)c);
    return s;
}

bool parse_logical(const std::string &v, int *out) {
    std::string s = lower(v);
    if (!s.empty() && s[0] == '.') s = s.substr(1);
    if (!s.empty() && (s[0] == 't')) { *out = 1; return true; }
    if (!s.empty() && (s[0] == 'f')) { *out = 0; return true; }
    return false;
}

bool parse_real(std::string v, double *out) {
    for (auto &c : v) if (c == 'd' || c == 'D') c = 'e';
    char *end = nullptr;
    double d = std::strtod(v.c_str(), &end);
    if (end == v.c_str()) return false;
    *out = d;
    return true;
}

}  // namespace

extern "C" int fp_parse_inp_text(const char *text, flite_controls *c, char *unknown,
                                 size_t unknown_len) {
    if (!text || !c) return FLITE_EINVAL;
    // strip comments, find the group body between '&' and '/'
    std::string s;
    {
        std::istringstream in(text);
        std::string line;
        while (std::getline(in, line)) {
            bool inq = false; char q = 0;
            std::string out;
            for (char ch : line) {
                if (inq) { out += ch; if (ch == q) inq = false; continue; }
                if (ch == '\'' || ch == '"') { inq = true; q = ch; out += ch; continue; }
                if (ch == '!') break;
                out += ch;
            }
            s += out + "\n";
        }
    }
    size_t amp = s.find('&');
    if (amp == std::string::npos) return FLITE_EIO;
    size_t p = amp + 1;
    while (p < s.size() && !std::isspace((unsigned char)s[p])) ++p;  // group name
    std::string unk;
    // tokenise "key = value" items
    while (p < s.size()) {
        while (p < s.size() && (std::isspace((unsigned char)s[p]) || s[p] == ',')) ++p;
        if (p >= s.size() || s[p] == '/') break;
        size_t eq = s.find('=', p);
        if (eq == std::string::npos) return FLITE_EIO;
        std::string key = s.substr(p, eq - p);
        while (!key.empty() && std::isspace((unsigned char)key.back())) key.pop_back();
        p = eq + 1;
        while (p < s.size() && std::isspace((unsigned char)s[p])) ++p;
        std::string val;
        if (p < s.size() && (s[p] == '\'' || s[p] == '"')) {
            char q = s[p++];
            size_t e = s.find(q, p);
            if (e == std::string::npos) return FLITE_EIO;
            val = s.substr(p, e - p);
            p = e + 1;
        } else {
            size_t e = p;
            while (e < s.size() && s[e] != ',' && s[e] != '\n' && s[e] != '/' &&
                   !std::isspace((unsigned char)s[e]))
                ++e;
            val = s.substr(p, e - p);
            p = e;
        }
        // strip the "ivd%" prefix
        std::string k = key;
        size_t pct = k.find('%');
        if (pct != std::string::npos) k = k.substr(pct + 1);
        std::string base = k, idx;
        size_t par = k.find('(');
        if (par != std::string::npos) { base = k.substr(0, par); idx = k.substr(par); }
        bool done = false;
        if (idx.empty()) {
            for (const Field &f : kFields) {
                if (!ieq(base, f.name)) continue;
                char *dst = (char *)c + f.off;
                if (f.kind == INT) {
                    double d; if (!parse_real(val, &d)) return FLITE_EIO;
                    *(int *)dst = (int)d;
                } else if (f.kind == DBL) {
                    double d; if (!parse_real(val, &d)) return FLITE_EIO;
                    *(double *)dst = d;
                } else {
                    int l; if (!parse_logical(val, &l)) return FLITE_EIO;
                    *(int *)dst = l;
                }
                done = true;
                break;
            }
        } else if (ieq(base, "datum") || ieq(base, "inflowField") || ieq(base, "enginesFrontMassFlow") ||
                   ieq(base, "enginesRearParameters")) {
            int i = 0, j = 1;
            if (std::sscanf(idx.c_str(), "(%d,%d)", &i, &j) < 1) return FLITE_EIO;
            double d; if (!parse_real(val, &d)) return FLITE_EIO;
            if (ieq(base, "datum") && i >= 1 && i <= 3) { c->datum[i - 1] = d; done = true; }
            if (ieq(base, "inflowField") && i >= 1 && i <= 6 && j >= 1 && j <= 2) {
                c->inflowField[(j - 1) * 6 + (i - 1)] = d; done = true;
            }
            if (ieq(base, "enginesFrontMassFlow") && i >= 1 && i <= 2) {
                c->enginesFrontMassFlow[i - 1] = d; done = true;
            }
            if (ieq(base, "enginesRearParameters") && i >= 1 && i <= 7 && j >= 1 && j <= 2) {
                c->enginesRearParameters[(j - 1) * 7 + (i - 1)] = d; done = true;
            }
        }
        if (!done) {
            if (!unk.empty()) unk += ",";
            unk += key;
        }
    }
    if (unknown && unknown_len) {
        std::snprintf(unknown, unknown_len, "%s", unk.c_str());
    }
    return FLITE_OK;
}

extern "C" int fp_read_inp(const char *path, flite_controls *c, char *unknown, size_t unknown_len) {
    if (!path) return FLITE_EINVAL;
    std::ifstream f(path);
    if (!f) return FLITE_EIO;
    std::stringstream ss;
    ss << f.rdbuf();
    std::string t = ss.str();
    return fp_parse_inp_text(t.c_str(), c, unknown, unknown_len);
}
