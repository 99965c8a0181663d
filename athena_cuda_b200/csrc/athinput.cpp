// athinput.cpp -- parameter files in the reference's athinput format
// (src/par.c): "<block>" headers, "name = value # comment" lines, '#' comment
// lines, "<par_end>" terminator, and "block/name=value" overrides that may only
// replace existing parameters (src/par.c:170-209).  Integer and real values are
// converted like atoi()/atof() (src/par.c:250-263).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "athb_internal.h"

struct athb_params {
  struct Par { std::string name, value; };
  struct Block { std::string name; std::vector<Par> pars; };
  std::vector<Block> blocks;

  Block* find_block(const std::string& n) {
    for (auto& b : blocks) if (b.name == n) return &b;
    return nullptr;
  }
  const Block* find_block(const std::string& n) const {
    for (auto& b : blocks) if (b.name == n) return &b;
    return nullptr;
  }
  const std::string* find(const char* block, const char* name) const {
    const Block* b = find_block(block);
    if (!b) return nullptr;
    for (auto& p : b->pars) if (p.name == name) return &p.value;
    return nullptr;
  }
};

static std::string trim(const std::string& s) {
  size_t a = 0, b = s.size();
  while (a < b && (s[a] == ' ' || s[a] == '\t' || s[a] == '\r' || s[a] == '\n')) a++;
  while (b > a && (s[b - 1] == ' ' || s[b - 1] == '\t' || s[b - 1] == '\r' || s[b - 1] == '\n')) b--;
  return s.substr(a, b - a);
}

static int parse_lines(const std::vector<std::string>& lines, const char* path, athb_params** out);

static std::vector<std::string> split_lines(const std::string& text) {
  std::vector<std::string> v;
  size_t a = 0;
  while (a <= text.size()) {
    size_t b = text.find('\n', a);
    if (b == std::string::npos) b = text.size();
    v.push_back(text.substr(a, b - a));
    a = b + 1;
  }
  return v;
}

extern "C" int athb_params_open(const char* path, athb_params** out) {
  if (!path || !out) return athb_fail(ATHB_ERR_ARG, "null argument");
  *out = nullptr;
  FILE* fp = fopen(path, "r");
  if (!fp) return athb_fail(ATHB_ERR_PARSE, "parameter file %s could not be opened", path);
  std::vector<std::string> lines;
  char line[1024];
  while (fgets(line, sizeof line, fp)) lines.push_back(line);
  fclose(fp);
  return parse_lines(lines, path, out);
}

extern "C" int athb_params_from_string(const char* text, athb_params** out) {
  if (!text || !out) return athb_fail(ATHB_ERR_ARG, "null argument");
  *out = nullptr;
  return parse_lines(split_lines(text), "<string>", out);
}

static int parse_lines(const std::vector<std::string>& lines, const char* path, athb_params** out) {
  athb_params* p = new athb_params();
  athb_params::Block* cur = nullptr;
  int lineno = 0;
  for (const std::string& raw : lines) {
    lineno++;
    std::string s = trim(raw);
    if (s.empty() || s[0] == '#') continue;
    if (s.compare(0, 9, "<par_end>") == 0) break;
    if (s[0] == '<') {
      size_t e = s.find('>');
      if (e == std::string::npos) {
        delete p;
        return athb_fail(ATHB_ERR_PARSE, "%s:%d: block name not terminated", path, lineno);
      }
      std::string name = trim(s.substr(1, e - 1));
      cur = p->find_block(name);
      if (!cur) { p->blocks.push_back({name, {}}); cur = &p->blocks.back(); }
      continue;
    }
    if (!cur) {
      delete p;
      return athb_fail(ATHB_ERR_PARSE, "%s:%d: parameter outside any <block>", path, lineno);
    }
    size_t hash = s.find('#');
    std::string body = hash == std::string::npos ? s : s.substr(0, hash);
    size_t eq = body.find('=');
    if (eq == std::string::npos) {
      delete p;
      return athb_fail(ATHB_ERR_PARSE, "%s:%d: no '=' in \"%s\"", path, lineno, s.c_str());
    }
    std::string name = trim(body.substr(0, eq)), value = trim(body.substr(eq + 1));
    bool replaced = false;
    for (auto& q : cur->pars) if (q.name == name) { q.value = value; replaced = true; }
    if (!replaced) cur->pars.push_back({name, value});
  }
  *out = p;
  return ATHB_OK;
}

extern "C" int athb_params_override(athb_params* p, const char* arg) {
  if (!p || !arg) return athb_fail(ATHB_ERR_ARG, "null argument");
  std::string s(arg);
  size_t sl = s.find('/');
  if (sl == std::string::npos) return ATHB_OK;  // not block/name=value: ignored, as src/par.c
  size_t eq = s.find('=', sl);
  if (eq == std::string::npos) return ATHB_OK;
  std::string block = s.substr(0, sl), name = s.substr(sl + 1, eq - sl - 1), value = s.substr(eq + 1);
  athb_params::Block* b = p->find_block(block);
  if (!b) return athb_fail(ATHB_ERR_NOTFOUND, "override: block \"%s\" not found", block.c_str());
  for (auto& q : b->pars)
    if (q.name == name) { q.value = value; return ATHB_OK; }
  return athb_fail(ATHB_ERR_NOTFOUND, "override: parameter \"%s\" not found", name.c_str());
}

extern "C" int athb_params_getd(const athb_params* p, const char* block, const char* name, double* v) {
  if (!p || !block || !name || !v) return athb_fail(ATHB_ERR_ARG, "null argument");
  const std::string* s = p->find(block, name);
  if (!s) return athb_fail(ATHB_ERR_NOTFOUND, "parameter %s/%s not found", block, name);
  *v = atof(s->c_str());
  return ATHB_OK;
}

extern "C" int athb_params_geti(const athb_params* p, const char* block, const char* name, int* v) {
  if (!p || !block || !name || !v) return athb_fail(ATHB_ERR_ARG, "null argument");
  const std::string* s = p->find(block, name);
  if (!s) return athb_fail(ATHB_ERR_NOTFOUND, "parameter %s/%s not found", block, name);
  *v = atoi(s->c_str());
  return ATHB_OK;
}

extern "C" const char* athb_params_gets(const athb_params* p, const char* block, const char* name) {
  const std::string* s = p ? p->find(block, name) : nullptr;
  return s ? s->c_str() : nullptr;
}

extern "C" void athb_params_close(athb_params* p) { delete p; }

// src/main.c:84-94 (time, gamma) and src/init_grid.c:25-120 (grid),
// src/set_bvals.c:163-257 (boundary flags).
extern "C" int athb_config_from_params(const athb_params* p, athb_config* cfg) {
  if (!p || !cfg) return athb_fail(ATHB_ERR_ARG, "null argument");
  athb_config c;
  memset(&c, 0, sizeof c);
  int rc = 0;
  rc |= athb_params_geti(p, "grid", "Nx1", &c.nx1);
  rc |= athb_params_geti(p, "grid", "Nx2", &c.nx2);
  rc |= athb_params_getd(p, "grid", "x1min", &c.x1min);
  rc |= athb_params_getd(p, "grid", "x1max", &c.x1max);
  rc |= athb_params_getd(p, "grid", "x2min", &c.x2min);
  rc |= athb_params_getd(p, "grid", "x2max", &c.x2max);
  rc |= athb_params_geti(p, "grid", "ibc_x1", &c.bc_ix1);
  rc |= athb_params_geti(p, "grid", "obc_x1", &c.bc_ox1);
  rc |= athb_params_geti(p, "grid", "ibc_x2", &c.bc_ix2);
  rc |= athb_params_geti(p, "grid", "obc_x2", &c.bc_ox2);
  rc |= athb_params_getd(p, "time", "cour_no", &c.cour_no);
  rc |= athb_params_getd(p, "time", "tlim", &c.tlim);
  rc |= athb_params_getd(p, "problem", "gamma", &c.gamma);
  if (rc) return ATHB_ERR_PARSE;
  if (athb_params_geti(p, "time", "nlim", &c.nlim) != ATHB_OK) c.nlim = -1;
  c.flux = ATHB_FLUX_ROE;
  if (const char* f = athb_params_gets(p, "job", "flux")) {
    if (!strcmp(f, "hlle")) c.flux = ATHB_FLUX_HLLE;
    else if (strcmp(f, "roe")) return athb_fail(ATHB_ERR_PARSE, "job/flux must be roe or hlle");
  }
  int dev = 0;
  if (athb_params_geti(p, "job", "device", &dev) == ATHB_OK) c.device = dev;
  *cfg = c;
  return athb_ctx_validate(&c);
}
