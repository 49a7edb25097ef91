// Host-side model construction for libufem_gpu.so: table checks, DOF
// numbering, block-sparse pattern, element colouring, element->block scatter
// map, supports/loads bookkeeping and the preparsed input reader.
//
// Reference interfaces restated here:
//   femReadInput           fem/fem_io.c:380-590 (preparsed variant, fem/feminput.5)
//   femReadInputLoads      fem/fem_io.c:86-165
//   fem_monte_read_data    fem/fem_mont.c:866-905
//   fem_dofs               fem/fem_sol.c:1263-1395
//   femKhit / femKpos      fem/fem_mloc.c:52-116
//   femMatPutAdd order     fem/fem_math.c:185-236 (first-touch column order)
//   fem_sol_res_alloc      fem/fem_sol.c:676-722 (reaction list)
//   femGetRepVal           fem/fem_accs.c:196-288 (value lookup by position)
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>
#include <mutex>

#include "ufem_internal.h"

namespace ufem {

static std::mutex g_err_mu;
static std::string g_err;

void set_error(const std::string &msg) {
  std::lock_guard<std::mutex> lk(g_err_mu);
  g_err = msg;
}

const char *last_error() {
  std::lock_guard<std::mutex> lk(g_err_mu);
  return g_err.c_str();
}

static int elem_nodes(long t) { return t == 2 ? 4 : 8; }
static int elem_dofs(long t) { return t == 2 ? 2 : 3; }

// Value of entry `idx` of a record, 0 when the record is shorter: the
// non-repeating branch of femGetRepVal (fem/fem_accs.c:236-252, :269-273).
static double rec_val(const std::vector<double> &rec, size_t idx) {
  return idx < rec.size() ? rec[idx] : 0.0;
}

int model_from_tables(const ufem_tables *t, ufem_model *m) {
  const auto t_start = std::chrono::steady_clock::now();
  if (!t || t->nLen < 2 || t->eLen < 1) {
    set_error("model tables: fewer than 2 nodes or no elements");
    return UFEM_AF_ERR_SML;  // fem/fem_io.c:516, :534
  }
  m->nLen = t->nLen;
  m->eLen = t->eLen;
  m->xyz.resize(3 * m->nLen);
  for (long i = 0; i < m->nLen; i++) {
    m->xyz[3 * i] = t->n_x[i];
    m->xyz[3 * i + 1] = t->n_y[i];
    m->xyz[3 * i + 2] = t->n_z ? t->n_z[i] : 0.0;
  }
  m->eType.assign(t->eType, t->eType + m->eLen);
  m->eRS.assign(t->eRS, t->eRS + m->eLen);
  m->eMP.assign(t->eMP, t->eMP + m->eLen);
  // element types: the quad (2) or the brick (9; 10 without Winkler springs)
  long t0 = m->eType[0];
  bool quad = (t0 == 2);
  for (long e = 0; e < m->eLen; e++) {
    long te = m->eType[e];
    bool ok = quad ? (te == 2) : (te == 9 || te == 10);
    if (!ok) {
      set_error("element types: only all-quad (2) or all-brick (9/10) models are on this path");
      return UFEM_AF_ERR_TYP;
    }
  }
  m->etype = quad ? 2 : 9;
  m->nn = elem_nodes(t0);
  m->b = elem_dofs(t0);
  m->enodes.resize((size_t)m->eLen * m->nn);
  for (long e = 0; e < m->eLen; e++) {
    // the caller's tables carry no length of eNodesL: every element but the
    // last is checked against the next element's start
    if (t->eFrom[e] < 0 || (e + 1 < m->eLen && t->eFrom[e + 1] - t->eFrom[e] != m->nn)) {
      set_error("element node count does not match its type");
      return UFEM_AF_ERR_SIZ;
    }
    for (int j = 0; j < m->nn; j++) {
      long np = t->eNodesL[t->eFrom[e] + j];
      if (np < 0 || np >= m->nLen) {
        set_error("invalid node position in element");  // fem/fem_sol.c:1304-1311
        return UFEM_AF_ERR_VAL;
      }
      m->enodes[(size_t)e * m->nn + j] = (int)np;
    }
  }
  // materials: type 1 (linear isotropic: DENS, EX, NU, ALPHA, KXX, C, PRICE,
  // fem/fem_m001.c:39) and type 5 (DENS, EX, NU, G, F_YC, F_YT, F_UC, F_UT,
  // fem/fem_m005.c:39; isotropic D, fem/fem_pl3d.c:190 and fem/fem_stf2.c:298)
  m->mpVals.resize(t->mpLen);
  m->mpTypeH.assign(t->mpType, t->mpType + t->mpLen);
  for (long p = 0; p < t->mpLen; p++) {
    long from = t->mpFrom[p];
    long to = (p + 1 < t->mpLen) ? t->mpFrom[p + 1] : t->mpLenL;
    if (from < 0 || to < from || to > t->mpLenL) {
      set_error("material value ranges out of order or out of range");
      return UFEM_AF_ERR_SIZ;
    }
    m->mpVals[p].assign(t->mpValL + from, t->mpValL + to);
  }
  m->eE.resize(m->eLen);
  m->eNu.resize(m->eLen);
  m->eThick.resize(m->eLen);
  m->eMat.resize(m->eLen);
  for (long e = 0; e < m->eLen; e++) {
    long p = m->eMP[e];
    if (p < 0 || p >= t->mpLen) {
      set_error("element material position out of range");
      return UFEM_AF_ERR_VAL;
    }
    if (t->mpType[p] != 1 && t->mpType[p] != 5) {
      set_error("material types: only linear isotropic (1, 5) is on this path");
      return UFEM_AF_ERR_TYP;
    }
    if (m->mpVals[p].size() > (t->mpType[p] == 5 ? 8u : 7u)) {
      // repeating values select the orthotropic plane D (fem/fem_stf2.c:256-266)
      set_error("materials with repeating values are not on this path");
      return UFEM_AF_ERR_TYP;
    }
    m->eMat[e] = p;
    m->eE[e] = rec_val(m->mpVals[p], 1);
    m->eNu[e] = rec_val(m->mpVals[p], 2);
    double thick = 0.0, winkler = 0.0;
    long r = m->eRS[e];
    if (t->rsLen > 0 && r >= 0 && r < t->rsLen) {
      long from = t->rsFrom[r];
      long to = (r + 1 < t->rsLen) ? t->rsFrom[r + 1] : t->rsLenL;
      if (from < 0 || to > t->rsLenL) {
        set_error("real set value ranges out of range");
        return UFEM_AF_ERR_SIZ;
      }
      if (to > from) {
        if (quad) thick = t->rsValL[from];       // RS_HEIGHT first, fem/fem_e002.c:1019
        else winkler = t->rsValL[from];          // RS_WINKLER, fem/fem_e010.c:79
      }
    }
    if (m->eType[e] == 10 && winkler > 0.0) {
      set_error("brick with Winkler foundation (type 10, RS_WINKLER > 0) is not on this path");
      return UFEM_AF_ERR_TYP;
    }
    m->eThick[e] = thick;
    if (quad && (m->eNu[e] <= 0.0 || m->eNu[e] >= 1.0)) {
      set_error("invalid Poisson ratio");  // fem/fem_stf2.c:47-54
      return UFEM_AF_ERR_VAL;
    }
  }
  // nodal loads and supports
  m->loads.clear();
  for (long i = 0; i < t->nlLen; i++) {
    NodalLoad l{t->nlNode[i], t->nlType[i], t->nlDir[i], t->nlVal[i]};
    if (l.node < 0 || l.node >= m->nLen) {
      set_error("load on an invalid node position");
      return UFEM_AF_ERR_VAL;
    }
    if (l.type != 1 && l.type != 3) {
      set_error("only supports (type 1) and nodal forces (type 3) are on this path");
      return UFEM_AF_ERR_TYP;
    }
    m->loads.push_back(l);
  }
  if (m->nID.empty()) {
    m->nID.resize(m->nLen);
    for (long i = 0; i < m->nLen; i++) m->nID[i] = i + 1;
  }
  if (m->eID.empty()) {
    m->eID.resize(m->eLen);
    for (long i = 0; i < m->eLen; i++) m->eID[i] = i + 1;
  }
  if (m->mpID.empty()) {
    m->mpID.resize(t->mpLen);
    for (long i = 0; i < t->mpLen; i++) m->mpID[i] = i + 1;
  }
  m->ms_ingest[2] = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count();
  return build_model(m);
}

int build_model(ufem_model *m) {
  // DOF numbering (fem_dofs, fem/fem_sol.c:1263), the block pattern
  // (femKhit, fem/fem_mloc.c:83), the scatter map and the element colouring
  // are built on the device
  auto t0 = std::chrono::steady_clock::now();
  int rv = gpu_build_pattern(m);
  if (rv != UFEM_AF_OK) return rv;
  auto t1 = std::chrono::steady_clock::now();
  if ((rv = setup_loads(m)) != UFEM_AF_OK) return rv;
  auto t2 = std::chrono::steady_clock::now();
  rv = upload_model(m);
  auto t3 = std::chrono::steady_clock::now();
  m->ms_ingest[3] = std::chrono::duration<double, std::milli>(t1 - t0).count();
  m->ms_ingest[4] = std::chrono::duration<double, std::milli>(t2 - t1).count();
  m->ms_ingest[5] = std::chrono::duration<double, std::milli>(t3 - t2).count();
  return rv;
}


// Loads and supports of the current tables: F after fem_add_loads
// (femApplyNLoad type 3: F[pos] += val, fem/fem_loads.c:343-395), the
// reaction list of fem_sol_res_alloc (fem/fem_sol.c:676-722) and the mask of
// zero-valued supports.
int setup_loads(ufem_model *m) {
  // ---- loads: F after fem_add_loads (femApplyNLoad type 3: F[pos] += val) ----
  m->F_loads.assign(m->nDOFAct, 0.0);
  m->has_nonzero_bc = false;
  m->reacNode.clear();
  m->reacDof.clear();
  m->reacRow.clear();
  m->fixedMask.assign(m->nDOFAct, 0);
  for (const auto &l : m->loads) {
    long p = (l.dir >= 1 && l.dir <= KNOWN_DOFS) ? m->dof(l.node * KNOWN_DOFS + l.dir - 1) : 0;
    if (l.type == 3) {
      if (p > 0) m->F_loads[p - 1] += l.val;
    } else if (l.type == 1) {
      if (p <= 0) {
        set_error("cannot add boundary condition on an unused DOF");  // fem/fem_loads.c:130-139
        return UFEM_AF_ERR_VAL;
      }
      if (l.val != 0.0) {
        m->has_nonzero_bc = true;
      } else {
        m->reacNode.push_back(l.node);
        m->reacDof.push_back(l.dir);
        m->reacRow.push_back((int)(p - 1));
        m->fixedMask[p - 1] = 1;
      }
    }
  }
  m->reacVal.assign(m->reacNode.size(), 0.0);
  return UFEM_AF_OK;
}

// The reference's row-slot K layout for this model, built on the host
// without any values: row sizes from femKhit (fem/fem_mloc.c:83-116), starts
// as in femMatAlloc (fem/fem_math.c:88-100) and columns in the order
// femLocKM_e/femMatPutAdd insert them (elements in order, local rows i, local
// columns j, a new column taking the first empty slot).
int export_rowslot(const ufem_model *m, long *frompos, long *defpos, long *pos, long *len) {
  const int nn = m->nn, b = m->b, s = nn * b;
  const long rows = m->nDOFAct;
  std::vector<long> krows(rows, 0);
  for (long e = 0; e < m->eLen; e++)
    for (int j = 0; j < nn; j++)
      for (int k = 0; k < b; k++) {
        long p = m->dof((long)m->enodes[(size_t)e * nn + j] * KNOWN_DOFS + k);
        if (p >= 1) krows[p - 1] += s;
      }
  long sum = 0;
  std::vector<long> from(rows);
  for (long i = 0; i < rows; i++) {
    sum += krows[i];
    from[i] = sum - krows[i];
  }
  if (len) *len = sum;
  if (frompos) std::copy(from.begin(), from.end(), frompos);
  if (defpos) std::copy(krows.begin(), krows.end(), defpos);
  if (!pos) return UFEM_AF_OK;
  std::fill(pos, pos + sum, 0L);
  std::vector<long> fill(rows, 0), lf(s);
  for (long e = 0; e < m->eLen; e++) {
    int q = 0;
    for (int j = 0; j < nn; j++)
      for (int k = 0; k < b; k++) lf[q++] = m->dof((long)m->enodes[(size_t)e * nn + j] * KNOWN_DOFS + k);
    for (int i = 0; i < s; i++) {
      long r = lf[i] - 1;
      for (int j = 0; j < s; j++) {
        long c = lf[j];
        long *row = pos + from[r];
        long f = fill[r];
        bool found = false;
        for (long t = 0; t < f; t++)
          if (row[t] == c) {
            found = true;
            break;
          }
        if (!found) {
          if (f >= krows[r]) {
            set_error("row-slot export: row overflow");
            return UFEM_AF_ERR_BIG;
          }
          row[f] = c;
          fill[r] = f + 1;
        }
      }
    }
  }
  return UFEM_AF_OK;
}

// ---------------------------------------------------------------------------
// preparsed input reader (femReadInput, fem/fem_io.c:380-590)
// ---------------------------------------------------------------------------
namespace {
struct Tok {
  const char *p, *end;
  bool ok = true;
  void skip() {
    while (p < end && (*p == ' ' || *p == '\n' || *p == '\t' || *p == '\r')) p++;
  }
  bool more() {
    skip();
    return p < end;
  }
  long L() {
    skip();
    if (p >= end) {
      ok = false;
      return 0;
    }
    char *q;
    long v = strtol(p, &q, 10);
    if (q == p) ok = false;
    p = q;
    return v;
  }
  double D() {
    skip();
    if (p >= end) {
      ok = false;
      return 0;
    }
    char *q;
    double v = strtod(p, &q);
    if (q == p) ok = false;
    p = q;
    return v;
  }
};
}  // namespace

namespace {

// The tables of an input file, as parsed from the text form or the binary
// form, before the model is built from them.
struct InputTables {
  std::vector<long> rsID, rsType, rsFrom;
  std::vector<double> rsVal;
  std::vector<long> mpID, mpType, mpFrom;
  std::vector<double> mpVal;
  std::vector<long> nID;
  std::vector<double> nx, ny, nz;
  std::vector<long> eID, eType, eRS, eMP, eFrom, eNodes;
  std::vector<long> nlNode, nlType, nlDir;
  std::vector<double> nlVal;
  long mc_ilen = 0, mc_olen = 0;
  std::vector<long> mc_pos, mc_type, mc_item, mc_sub, mc_iter;
};

int parse_text(const std::string &buf, InputTables &in) {
  Tok t{buf.data(), buf.data() + buf.size()};
  // solution control data (fem/fem_io.c:408-414)
  t.L(); t.L();
  t.L(); t.L(); t.L();
  // real sets (fem/fem_io.c:421-475)
  long rsLen = t.L();
  long sum = 0;
  for (long i = 0; i < rsLen; i++) {
    in.rsID.push_back(t.L());
    in.rsType.push_back(t.L());
    long c = t.L();
    in.rsFrom.push_back(sum);
    sum += c;
  }
  if (rsLen > 0) {
    long rsLenL = t.L();
    if (rsLenL != sum) {
      set_error("bad number of real set values");
      return UFEM_AF_ERR_SIZ;
    }
    for (long i = 0; i < rsLenL; i++) in.rsVal.push_back(t.D());
  }
  // materials (fem/fem_io.c:478-521)
  long mpLen = t.L();
  sum = 0;
  for (long i = 0; i < mpLen; i++) {
    in.mpID.push_back(t.L());
    in.mpType.push_back(t.L());
    long c = t.L();
    in.mpFrom.push_back(sum);
    sum += c;
  }
  if (mpLen > 0) {
    long mpLenL = t.L();
    if (mpLenL != sum) {
      set_error("bad number of material property values");
      return UFEM_AF_ERR_SIZ;
    }
    for (long i = 0; i < mpLenL; i++) in.mpVal.push_back(t.D());
  }
  // nodes (fem/fem_io.c:524-540)
  long nLen = t.L();
  if (nLen < 2) {
    set_error("fewer than 2 nodes");
    return UFEM_AF_ERR_SML;
  }
  in.nID.resize(nLen);
  in.nx.resize(nLen);
  in.ny.resize(nLen);
  in.nz.resize(nLen);
  for (long i = 0; i < nLen; i++) {
    in.nID[i] = t.L();
    in.nx[i] = t.D();
    in.ny[i] = t.D();
    in.nz[i] = t.D();
  }
  // elements (fem/fem_io.c:543-598)
  long eLen = t.L();
  if (eLen < 1) {
    set_error("no elements");
    return UFEM_AF_ERR_SML;
  }
  in.eID.resize(eLen);
  in.eType.resize(eLen);
  in.eRS.resize(eLen);
  in.eMP.resize(eLen);
  in.eFrom.resize(eLen);
  sum = 0;
  for (long i = 0; i < eLen; i++) {
    in.eID[i] = t.L();
    in.eType[i] = t.L();
    in.eRS[i] = t.L();
    in.eMP[i] = t.L();
    long c = t.L();
    in.eFrom[i] = sum;
    sum += c;
  }
  long eLenL = t.L();
  if (eLenL != sum) {
    set_error("bad number of element nodes");
    return UFEM_AF_ERR_SIZ;
  }
  in.eNodes.resize(eLenL);
  for (long i = 0; i < eLenL; i++) in.eNodes[i] = t.L();
  // gravity (fem/fem_io.c:604) -- only zero gravity is on this path
  t.L();
  double grVal = t.D();
  if (std::fabs(grVal) > 0) {
    set_error("gravity loads are not on this path");
    return UFEM_AF_ERR_TYP;
  }
  // nodal loads (fem/fem_io.c:92-113)
  long nlLen = t.L();
  in.nlNode.resize(nlLen);
  in.nlType.resize(nlLen);
  in.nlDir.resize(nlLen);
  in.nlVal.resize(nlLen);
  for (long i = 0; i < nlLen; i++) {
    in.nlNode[i] = t.L();
    in.nlType[i] = t.L();
    in.nlDir[i] = t.L();
    in.nlVal[i] = t.D();
  }
  // element loads (fem/fem_io.c:116) -- none on this path
  long elLen = t.L();
  if (elLen > 0) {
    set_error("element loads are not on this path");
    return UFEM_AF_ERR_TYP;
  }
  if (!t.ok) {
    set_error("truncated input file");
    return UFEM_AF_ERR_IO;
  }
  // transient and dynamics counters (fem/fem_io.c:176, :297) and the
  // optional Monte Carlo table (fem/fem_mont.c:873-905)
  if (t.more()) {
    long transNum = t.L(), dynNum = t.L();
    t.D();
    if (dynNum > 0 && transNum > 0) {
      set_error("transient data are not on this path");
      return UFEM_AF_ERR_TYP;
    }
    if (t.more()) {
      long dynNum0 = t.L();
      if (dynNum0 > 0) {
        set_error("dynamics data are not on this path");
        return UFEM_AF_ERR_TYP;
      }
      if (t.more()) {
        long ilen = t.L(), olen = t.L();
        if (t.ok && ilen > 0) {
          in.mc_ilen = ilen;
          in.mc_olen = olen;
          for (long i = 0; i < ilen + olen; i++) {
            in.mc_pos.push_back(t.L());
            in.mc_type.push_back(t.L());
            in.mc_item.push_back(t.L());
            in.mc_sub.push_back(t.L());
            in.mc_iter.push_back(t.L());
          }
          if (!t.ok) {
            set_error("incomplete or unavailable random data");  // fem/fem_mont.c:885
            return UFEM_AF_ERR_IO;
          }
        }
      }
    }
  }
  return UFEM_AF_OK;
}

// ---- binary form (no reference counterpart) --------------------------------
// "UFEMBIN1", a uint32 byte-order mark 0x01020304, then 28 arrays, each as an
// int64 count followed by count little-endian int64 (integer tables) or
// float64 (coordinates and values) items, in the order of kBinOrder below.
// The MC table's ilen and olen travel as a 2-item array.
constexpr char kBinMagic[8] = {'U', 'F', 'E', 'M', 'B', 'I', 'N', '1'};
constexpr uint32_t kBinBom = 0x01020304u;

struct BinArray {
  std::vector<long> *l;
  std::vector<double> *d;
};

std::vector<BinArray> bin_order(InputTables &in, std::vector<long> &mc_len) {
  return {{&in.rsID, nullptr},   {&in.rsType, nullptr}, {&in.rsFrom, nullptr}, {nullptr, &in.rsVal},
          {&in.mpID, nullptr},   {&in.mpType, nullptr}, {&in.mpFrom, nullptr}, {nullptr, &in.mpVal},
          {&in.nID, nullptr},    {nullptr, &in.nx},     {nullptr, &in.ny},     {nullptr, &in.nz},
          {&in.eID, nullptr},    {&in.eType, nullptr},  {&in.eRS, nullptr},    {&in.eMP, nullptr},
          {&in.eFrom, nullptr},  {&in.eNodes, nullptr}, {&in.nlNode, nullptr}, {&in.nlType, nullptr},
          {&in.nlDir, nullptr},  {nullptr, &in.nlVal},  {&mc_len, nullptr},    {&in.mc_pos, nullptr},
          {&in.mc_type, nullptr}, {&in.mc_item, nullptr}, {&in.mc_sub, nullptr}, {&in.mc_iter, nullptr}};
}

bool is_binary(const std::string &buf) {
  return buf.size() >= sizeof(kBinMagic) && std::memcmp(buf.data(), kBinMagic, sizeof(kBinMagic)) == 0;
}

int parse_binary(const std::string &buf, InputTables &in) {
  static_assert(sizeof(long) == 8 && sizeof(double) == 8, "64-bit long and double");
  size_t off = sizeof(kBinMagic);
  uint32_t bom = 0;
  if (buf.size() < off + sizeof(bom)) {
    set_error("truncated binary input");
    return UFEM_AF_ERR_IO;
  }
  std::memcpy(&bom, buf.data() + off, sizeof(bom));
  off += sizeof(bom);
  if (bom != kBinBom) {
    set_error("binary input written with another byte order");
    return UFEM_AF_ERR_IO;
  }
  std::vector<long> mc_len;
  for (BinArray &a : bin_order(in, mc_len)) {
    int64_t n = 0;
    if (buf.size() - off < sizeof(n)) {
      set_error("truncated binary input");
      return UFEM_AF_ERR_IO;
    }
    std::memcpy(&n, buf.data() + off, sizeof(n));
    off += sizeof(n);
    if (n < 0 || (uint64_t)n > (buf.size() - off) / 8) {
      set_error("truncated binary input");
      return UFEM_AF_ERR_IO;
    }
    // one copy pass (the array may sit at any byte offset of the file)
    if (a.l) {
      a.l->clear();
      a.l->reserve(n);
      const char *src = buf.data() + off;
      for (int64_t i = 0; i < n; i += 4096) {
        long tmp[4096];
        const int64_t c = std::min<int64_t>(4096, n - i);
        std::memcpy(tmp, src + i * 8, c * 8);
        a.l->insert(a.l->end(), tmp, tmp + c);
      }
    } else {
      a.d->clear();
      a.d->reserve(n);
      const char *src = buf.data() + off;
      for (int64_t i = 0; i < n; i += 4096) {
        double tmp[4096];
        const int64_t c = std::min<int64_t>(4096, n - i);
        std::memcpy(tmp, src + i * 8, c * 8);
        a.d->insert(a.d->end(), tmp, tmp + c);
      }
    }
    off += n * 8;
  }
  // the shapes the text reader would have produced
  const size_t nLen = in.nID.size(), eLen = in.eID.size();
  bool ok = in.rsType.size() == in.rsID.size() && in.rsFrom.size() == in.rsID.size() &&
            in.mpType.size() == in.mpID.size() && in.mpFrom.size() == in.mpID.size() && in.nx.size() == nLen &&
            in.ny.size() == nLen && in.nz.size() == nLen && in.eType.size() == eLen && in.eRS.size() == eLen &&
            in.eMP.size() == eLen && in.eFrom.size() == eLen && in.nlType.size() == in.nlNode.size() &&
            in.nlDir.size() == in.nlNode.size() && in.nlVal.size() == in.nlNode.size() && mc_len.size() == 2;
  for (size_t i = 0; ok && i < eLen; i++)
    ok = in.eFrom[i] >= 0 && in.eFrom[i] <= (long)in.eNodes.size() && (i == 0 || in.eFrom[i] >= in.eFrom[i - 1]);
  for (size_t i = 0; ok && i < in.rsFrom.size(); i++) ok = in.rsFrom[i] >= 0 && in.rsFrom[i] <= (long)in.rsVal.size();
  for (size_t i = 0; ok && i < in.mpFrom.size(); i++) ok = in.mpFrom[i] >= 0 && in.mpFrom[i] <= (long)in.mpVal.size();
  if (ok) {
    in.mc_ilen = mc_len[0];
    in.mc_olen = mc_len[1];
    const size_t nmc = in.mc_ilen > 0 ? (size_t)(in.mc_ilen + in.mc_olen) : 0;
    ok = in.mc_ilen >= 0 && in.mc_olen >= 0 && in.mc_pos.size() == nmc && in.mc_type.size() == nmc &&
         in.mc_item.size() == nmc && in.mc_sub.size() == nmc && in.mc_iter.size() == nmc;
  }
  if (!ok) {
    set_error("inconsistent binary input");
    return UFEM_AF_ERR_SIZ;
  }
  if (nLen < 2) {
    set_error("fewer than 2 nodes");
    return UFEM_AF_ERR_SML;
  }
  if (eLen < 1) {
    set_error("no elements");
    return UFEM_AF_ERR_SML;
  }
  return UFEM_AF_OK;
}

int write_binary(InputTables &in, const char *fname) {
  std::ofstream f(fname, std::ios::binary | std::ios::trunc);
  if (!f) {
    set_error(std::string("cannot open output ") + fname);
    return UFEM_AF_ERR_IO;
  }
  f.write(kBinMagic, sizeof(kBinMagic));
  f.write(reinterpret_cast<const char *>(&kBinBom), sizeof(kBinBom));
  std::vector<long> mc_len = {in.mc_ilen, in.mc_olen};
  for (BinArray &a : bin_order(in, mc_len)) {
    const int64_t n = a.l ? (int64_t)a.l->size() : (int64_t)a.d->size();
    f.write(reinterpret_cast<const char *>(&n), sizeof(n));
    if (n) f.write(a.l ? reinterpret_cast<const char *>(a.l->data()) : reinterpret_cast<const char *>(a.d->data()),
                   n * 8);
  }
  if (!f) {
    set_error(std::string("cannot write ") + fname);
    return UFEM_AF_ERR_IO;
  }
  return UFEM_AF_OK;
}

// Shape checks shared by both readers, before any table is indexed: every
// quad (4 nodes) and brick (8 nodes) element holds exactly its node count in
// the element-node list (a truncated list or a miscounted element would make
// model_from_tables read past it), and the real-set and material value
// ranges start in order inside their value lists.
int check_tables(const InputTables &in) {
  const long eLen = (long)in.eFrom.size(), eLenL = (long)in.eNodes.size();
  for (long e = 0; e < eLen; e++) {
    const long from = in.eFrom[e], to = e + 1 < eLen ? in.eFrom[e + 1] : eLenL;
    if (from < 0 || to < from || to > eLenL) {
      set_error("element node list out of order or out of range");
      return UFEM_AF_ERR_SIZ;
    }
    const long te = in.eType[e];
    if ((te == 2 || te == 9 || te == 10) && to - from != elem_nodes(te)) {
      set_error("element " + std::to_string(e) + " of type " + std::to_string(te) + " has " +
                std::to_string(to - from) + " nodes, not " + std::to_string(elem_nodes(te)));
      return UFEM_AF_ERR_SIZ;
    }
  }
  auto ranges_ok = [](const std::vector<long> &from, size_t nvals) {
    for (size_t i = 0; i < from.size(); i++) {
      const long next = i + 1 < from.size() ? from[i + 1] : (long)nvals;
      if (from[i] < 0 || next < from[i] || next > (long)nvals) return false;
    }
    return true;
  };
  if (!ranges_ok(in.rsFrom, in.rsVal.size()) || !ranges_ok(in.mpFrom, in.mpVal.size())) {
    set_error("real set or material value ranges out of order or out of range");
    return UFEM_AF_ERR_SIZ;
  }
  return UFEM_AF_OK;
}

// the whole file in one buffer, read with one pass of read(2)
int read_file(const char *fname, std::string &buf) {
  const int fd = ::open(fname, O_RDONLY);
  struct stat st;
  if (fd < 0 || ::fstat(fd, &st) != 0) {
    if (fd >= 0) ::close(fd);
    set_error(std::string("cannot open input ") + fname);
    return UFEM_AF_ERR_IO;
  }
  buf.resize((size_t)st.st_size);
  size_t got = 0;
  while (got < buf.size()) {
    const ssize_t r = ::read(fd, &buf[got], buf.size() - got);
    if (r <= 0) break;
    got += (size_t)r;
  }
  ::close(fd);
  if (got != buf.size()) {
    set_error(std::string("cannot read input ") + fname);
    return UFEM_AF_ERR_IO;
  }
  return UFEM_AF_OK;
}

}  // namespace

int read_input_file(const char *fname, ufem_model **out) {
  const auto t0 = std::chrono::steady_clock::now();
  std::string buf;
  int rv = read_file(fname, buf);
  if (rv != UFEM_AF_OK) return rv;
  const auto t1 = std::chrono::steady_clock::now();
  InputTables in;
  rv = is_binary(buf) ? parse_binary(buf, in) : parse_text(buf, in);
  if (rv != UFEM_AF_OK) return rv;
  if ((rv = check_tables(in)) != UFEM_AF_OK) return rv;
  const auto t2 = std::chrono::steady_clock::now();
  ufem_model *m = new ufem_model();
  m->ms_ingest[0] = std::chrono::duration<double, std::milli>(t1 - t0).count();
  m->ms_ingest[1] = std::chrono::duration<double, std::milli>(t2 - t1).count();
  m->mc_ilen = in.mc_ilen;
  m->mc_olen = in.mc_olen;
  m->mc_pos = in.mc_pos;
  m->mc_type = in.mc_type;
  m->mc_item = in.mc_item;
  m->mc_sub = in.mc_sub;
  m->mc_iter = in.mc_iter;
  m->nID = in.nID;
  m->eID = in.eID;
  m->mpID = in.mpID;
  m->rsID = in.rsID;
  ufem_tables tb{};
  tb.nLen = (long)in.nID.size(); tb.n_x = in.nx.data(); tb.n_y = in.ny.data(); tb.n_z = in.nz.data();
  tb.eLen = (long)in.eID.size(); tb.eType = in.eType.data(); tb.eRS = in.eRS.data(); tb.eMP = in.eMP.data();
  tb.eFrom = in.eFrom.data(); tb.eNodesL = in.eNodes.data();
  tb.rsLen = (long)in.rsID.size(); tb.rsType = in.rsType.data(); tb.rsFrom = in.rsFrom.data();
  tb.rsLenL = (long)in.rsVal.size(); tb.rsValL = in.rsVal.data();
  tb.mpLen = (long)in.mpID.size(); tb.mpType = in.mpType.data(); tb.mpFrom = in.mpFrom.data();
  tb.mpLenL = (long)in.mpVal.size(); tb.mpValL = in.mpVal.data();
  tb.nlLen = (long)in.nlNode.size(); tb.nlNode = in.nlNode.data(); tb.nlType = in.nlType.data();
  tb.nlDir = in.nlDir.data(); tb.nlVal = in.nlVal.data();
  rv = model_from_tables(&tb, m);
  if (rv != UFEM_AF_OK) {
    delete m;
    return rv;
  }
  *out = m;
  return UFEM_AF_OK;
}

int convert_input_file(const char *text_fname, const char *bin_fname) {
  std::string buf;
  int rv = read_file(text_fname, buf);
  if (rv != UFEM_AF_OK) return rv;
  InputTables in;
  if ((rv = is_binary(buf) ? parse_binary(buf, in) : parse_text(buf, in)) != UFEM_AF_OK) return rv;
  if ((rv = check_tables(in)) != UFEM_AF_OK) return rv;
  return write_binary(in, bin_fname);
}

}  // namespace ufem
