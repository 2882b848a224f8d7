/*
 * Test infrastructure (oracle build only): a command-line driver written for
 * this repository that runs the reference library (mcbapo/mpsdyn, compiled
 * from source into oracle/_ref by oracle/Makefile) on files written by the
 * tests.  Inputs and outputs use the reference's own binary formats:
 * mwArray = int rank, int dims[rank], double data[2n] column-major re/im
 * (src/wrapper/mwArray.cpp:382-442); MPS = int length, int bond, double
 * normfact, int gauge, then per site int pos + mwArray
 * (src/core/cpp/MPS.cpp:442-509, src/core/cpp/Site.cpp:561-578).
 * Scalars are printed as one JSON object on the last line of stdout.
 *
 * Models are given as one argument:
 *   ising:L:J:g:h              IsingHamiltonian(L,2,J,g,h)   (IsingHamiltonian.cpp:17-29)
 *   schwinger:N:mu:x:l0:alpha  SchwingerHamiltonian(N,mu,x,l0,alpha)  (SchwingerHamiltonian.cpp:13-21)
 *
 * Commands (each maps onto one reference call path):
 *   matvec L W R x y [offset]      TensorMultiplierOffset::product   (TensorMultiplierOffset.cpp:14-17)
 *   matvec_herm L W R x y          TensorMultiplierHermitian::product (TensorMultiplierHermitian.cpp:37-70)
 *   envL Lold ket W bra out        Operator::contractL                (Operator.cpp:273-334)
 *   envR Rold ket W bra out        Operator::contractR                (Operator.cpp:336-398)
 *   mpo model prefix               writes W_k of getHMPO as prefix<k>.bin
 *   umpo model delta imag prefix   writes W_k of IsingHamiltonian::getUMPO (IsingHamiltonian.cpp:131-148)
 *   energy model mps               Contractor::contract(mps,H,mps)    (Contractor.cpp:528-556)
 *   gs model D convtol eigtol init out
 *                                  Contractor::findGroundState        (Contractor.cpp:1352-1533)
 *   exc model D convtol eigtol init0 init1 out0 out1
 *                                  findGroundState + findNextExcitedState (Contractor.cpp:2676-2727)
 *   imag model D M delta convtol [init]
 *                                  testIsing imaginary-time loop (programs/ising/testIsing.cpp:106-138)
 *   evolve model D M dt convtol init out
 *                                  flatIsing real-time loop (programs/banulsm/curved/flatIsing.cpp:174-205):
 *                                  per step <sigma_x>_k, energy and centre entropy
 *   expect mps op                  <op_k> for every site, op in {sx,sy,sz} (flatIsing.cpp:258-282)
 *   entropy mps pos                Contractor::getEntropy             (Contractor.cpp:2045-2076)
 *   schmidt mps pos                Contractor::getSchmidtValues       (Contractor.cpp:2243-2270)
 *   truncate mps D out             MPS(mps, D) (SVD cut, MPS.cpp:761-772)
 *   contract2 model mps            Contractor::contract2(H, mps) = <mps|H^dag H|mps> (Contractor.cpp:634-653)
 *   opterr model delta imag D mps  one Contractor::optimize step with errN, errT (Contractor.cpp:263-276)
 *   applympo model delta imag D dagger dir mps out
 *                                  U-MPO of getUMPO applied to mps: MPS::applyExactly (D = 0) or
 *                                  MPS::approximate (D > 0), MPS.cpp:853-936
 *   profile model D eigtol init n [pos0]
 *                                  timed sample: n site steps of the ground-state sweep
 *                                  from site pos0 (default: around the chain centre),
 *                                  the CPU baseline of the bench
 *   gauge mps dir out              MPS::gaugeCond(dir, true)          (MPS.cpp:306-364)
 *   savempo model file             MPO::saveMPO of the model's H     (MPO.cpp:214-231)
 *   optsum D convtol init out ket re im [ket re im ...]
 *                                  Contractor::optimizeSum            (Contractor.cpp:2332-2477)
 */
#include "Contractor.h"
#include "IsingHamiltonian.h"
#include "SchwingerHamiltonian.h"
#include "HeisenbergHamiltonian.h"
#include "BoseHubbardHamiltonian.h"
#include "MPS.h"
#include "MPO.h"
#include "Operator.h"
#include "Site.h"
#include "TensorMultiplierOffset.h"
#include "TensorMultiplierHermitian.h"
#include "mwArray.h"
#include "Indices.h"
#include "wrapper.h"
#include <ctime>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

using namespace std;
using namespace shrt;

// Counters of the eigensolver shim (oracle/eigs_shim.cpp).
extern long long g_shim_products;
extern long long g_shim_solves;

namespace {

double now_s() {
  struct timespec t;
  clock_gettime(CLOCK_MONOTONIC, &t);
  return t.tv_sec + 1e-9 * t.tv_nsec;
}

mwArray load_array(const char* fn) {
  ifstream in(fn, ios::binary);
  if (!in.is_open()) { cerr << "cannot open " << fn << endl; exit(3); }
  mwArray a;
  a.load(in);
  return a;
}

void save_array(const mwArray& a, const char* fn) {
  ofstream out(fn, ios::binary);
  a.save(out);
}

vector<string> split(const string& s, char c) {
  vector<string> out;
  stringstream ss(s);
  string item;
  while (getline(ss, item, c)) out.push_back(item);
  return out;
}

struct Model {
  IsingHamiltonian* ising = nullptr;
  SchwingerHamiltonian* schw = nullptr;
  HeisenbergHamiltonian* heis = nullptr;
  BoseHubbardHamiltonian* bh = nullptr;
  int L = 0;
  const MPO& H() {
    return ising ? ising->getHMPO(0.) : heis ? heis->getHMPO() : bh ? bh->getHMPO() : schw->getHMPO();
  }
};

Model make_model(const char* spec) {
  vector<string> p = split(spec, ':');
  Model m;
  if (p[0] == "ising") {
    m.L = atoi(p[1].c_str());
    m.ising = new IsingHamiltonian(m.L, 2, atof(p[2].c_str()), atof(p[3].c_str()),
                                   atof(p[4].c_str()));
  } else if (p[0] == "schwinger") {
    m.L = atoi(p[1].c_str());
    m.schw = new SchwingerHamiltonian(m.L, atof(p[2].c_str()), atof(p[3].c_str()),
                                      atof(p[4].c_str()), atof(p[5].c_str()));
  } else if (p[0] == "heis") {
    // heis:L:Jx:Jy:Jz:hx:hy:hz:offset  (HeisenbergHamiltonian.cpp, d = 2)
    m.L = atoi(p[1].c_str());
    m.heis = new HeisenbergHamiltonian(m.L, atof(p[2].c_str()), atof(p[3].c_str()), atof(p[4].c_str()),
                                       atof(p[5].c_str()), atof(p[6].c_str()), atof(p[7].c_str()), 2,
                                       atof(p[8].c_str()));
  } else if (p[0] == "bh") {
    // bh:L:N:t:U:Ntarget:penN:V  (BoseHubbardHamiltonian.cpp, uniform couplings, d = N + 1)
    m.L = atoi(p[1].c_str());
    m.bh = new BoseHubbardHamiltonian(m.L, atoi(p[2].c_str()), atof(p[3].c_str()), atof(p[4].c_str()),
                                      atoi(p[5].c_str()), atof(p[6].c_str()), atof(p[7].c_str()));
  } else {
    cerr << "unknown model " << spec << endl;
    exit(3);
  }
  return m;
}

void print_json(const vector<pair<string, double> >& kv,
                const vector<pair<string, vector<double> > >& arrays = {}) {
  printf("{");
  bool first = true;
  for (auto& e : kv) {
    printf("%s\"%s\": %.17g", first ? "" : ", ", e.first.c_str(), e.second);
    first = false;
  }
  for (auto& e : arrays) {
    printf("%s\"%s\": [", first ? "" : ", ", e.first.c_str());
    for (size_t i = 0; i < e.second.size(); i++)
      printf("%s%.17g", i ? ", " : "", e.second[i]);
    printf("]");
    first = false;
  }
  printf("}\n");
  fflush(stdout);
}

// <op_k> for every site, as flatIsing.cpp:258-282 computes it.
vector<double> expectations(const MPS& state, const mwArray& op2) {
  Contractor& c = Contractor::theContractor();
  int len = state.getLength();
  int d = 2;
  mwArray id_ = identityMatrix(d);
  id_.reshape(Indices(d, 1, d, 1));
  Operator ident(id_);
  mwArray o = op2;
  o.reshape(Indices(d, 1, d, 1));
  Operator oper(o);
  MPO ops(len);
  for (int k = 0; k < len; k++) ops.setOp(k, &ident, false);
  double nrm = real(c.contract(state, state));
  vector<double> out;
  for (int pos = 0; pos < len; pos++) {
    ops.setOp(pos, &oper, false);
    out.push_back(real(c.contract(state, ops, state)) / nrm);
    ops.setOp(pos, &ident, false);
  }
  return out;
}

mwArray pauli(const string& name) {
  complex_t dx[] = {ZERO_c, ONE_c, ONE_c, ZERO_c};
  complex_t dy[] = {ZERO_c, I_c, -1. * I_c, ZERO_c};
  complex_t dz[] = {ONE_c, ZERO_c, ZERO_c, -1. * ONE_c};
  if (name == "sx") return mwArray(Indices(2, 2), dx);
  if (name == "sy") return mwArray(Indices(2, 2), dy);
  return mwArray(Indices(2, 2), dz);
}

}  // namespace

int main(int argc, const char* argv[]) {
  if (argc < 2) { cerr << "usage: ref_driver <command> ..." << endl; return 2; }
  string cmd = argv[1];
  cout.precision(17);
  Contractor& contractor = Contractor::theContractor();

  if (cmd == "matvec" || cmd == "matvec_herm") {
    mwArray L = load_array(argv[2]), W = load_array(argv[3]), R = load_array(argv[4]);
    mwArray x = load_array(argv[5]);
    double offset = argc > 7 ? atof(argv[7]) : 0.;
    mwArray y;
    x.reshape(Indices(-1, 1));
    if (cmd == "matvec") {
      TensorMultiplierOffset m(L, W, R, offset);
      m.product(x, y);
    } else {
      TensorMultiplierHermitian m(L, W, R);
      m.product(x, y);
    }
    save_array(y, argv[6]);
    print_json({{"n", (double)y.getNrComponents()}});
  } else if (cmd == "envL" || cmd == "envR") {
    mwArray T = load_array(argv[2]), ket = load_array(argv[3]);
    mwArray W = load_array(argv[4]), bra = load_array(argv[5]);
    Operator op(W);
    Site sk(0, ket), sb(0, bra);
    mwArray out;
    if (cmd == "envL") op.contractL(out, T, sk, sb);
    else op.contractR(out, T, sk, sb);
    save_array(out, argv[6]);
    print_json({{"n", (double)out.getNrComponents()}});
  } else if (cmd == "mpo") {
    Model m = make_model(argv[2]);
    const MPO& H = m.H();
    for (int k = 0; k < m.L; k++) {
      string fn = string(argv[3]) + to_string(k) + ".bin";
      save_array(H.getOp(k).getFullData(), fn.c_str());
    }
    print_json({{"L", (double)m.L}});
  } else if (cmd == "umpo") {
    Model m = make_model(argv[2]);
    MPO U(m.L);
    m.ising->getUMPO(U, atof(argv[3]), 0., atoi(argv[4]) != 0, 2);
    for (int k = 0; k < m.L; k++) {
      string fn = string(argv[5]) + to_string(k) + ".bin";
      save_array(U.getOp(k).getFullData(), fn.c_str());
    }
    print_json({{"L", (double)m.L}});
  } else if (cmd == "energy") {
    Model m = make_model(argv[2]);
    MPS s;
    s.importMPS(argv[3]);
    complex_t e = contractor.contract(s, m.H(), s);
    complex_t n = contractor.contract(s, s);
    print_json({{"E_re", e.re}, {"E_im", e.im}, {"norm_re", n.re}});
  } else if (cmd == "contract2") {
    Model m = make_model(argv[2]);
    MPS s;
    s.importMPS(argv[3]);
    complex_t v = contractor.contract2(m.H(), s);
    print_json({{"re", v.re}, {"im", v.im}});
  } else if (cmd == "opterr") {
    Model m = make_model(argv[2]);
    MPO U(m.L);
    m.ising->getUMPO(U, atof(argv[3]), 0., atoi(argv[4]) != 0, 2);
    contractor.setConvTol(1e-10);
    MPS orig;
    orig.importMPS(argv[6]);
    MPS init(orig);
    double errN = 0., errT = 0.;
    contractor.optimize(U, orig, init, atoi(argv[5]), &errN, &errT);
    print_json({{"errN", errN}, {"errT", errT}, {"normfact", init.getNormFact()}});
  } else if (cmd == "gs") {
    Model m = make_model(argv[2]);
    int D = atoi(argv[3]);
    contractor.setConvTol(atof(argv[4]));
    contractor.setEigTol(atof(argv[5]));
    MPS gs;
    gs.importMPS(argv[6]);
    double E0 = 0;
    double t0 = now_s();
    contractor.findGroundState(m.H(), D, &E0, gs);
    double t1 = now_s();
    gs.exportMPS(argv[7]);
    print_json({{"E0", E0}, {"seconds", t1 - t0}, {"products", (double)g_shim_products},
                {"site_solves", (double)g_shim_solves}});
  } else if (cmd == "exc") {
    Model m = make_model(argv[2]);
    int D = atoi(argv[3]);
    contractor.setConvTol(atof(argv[4]));
    contractor.setEigTol(atof(argv[5]));
    MPS gs, exc;
    gs.importMPS(argv[6]);
    exc.importMPS(argv[7]);
    double E0 = 0, E1 = 0;
    double t0 = now_s();
    contractor.findGroundState(m.H(), D, &E0, gs);
    double t1 = now_s();
    long long p0 = g_shim_products, s0 = g_shim_solves;
    gs.exportMPS(argv[8]);
    vector<MPS*> levels(1, &gs);
    contractor.findNextExcitedState(m.H(), D, levels, &E1, exc);
    double t2 = now_s();
    exc.exportMPS(argv[9]);
    complex_t ov = contractor.contract(exc, gs);
    print_json({{"E0", E0}, {"E1", E1}, {"gap", E1 - E0}, {"overlap_abs", abs(ov)},
                {"gs_seconds", t1 - t0}, {"exc_seconds", t2 - t1},
                {"gs_products", (double)p0}, {"gs_site_solves", (double)s0},
                {"exc_products", (double)(g_shim_products - p0)},
                {"exc_site_solves", (double)(g_shim_solves - s0)}});
  } else if (cmd == "imag") {
    Model m = make_model(argv[2]);
    int D = atoi(argv[3]);
    int M = atoi(argv[4]);
    double delta = atof(argv[5]);
    contractor.setConvTol(atof(argv[6]));
    int L = m.L, d = 2;
    MPS state(L, D, d);
    if (argc > 7) state.importMPS(argv[7]);
    MPO evol(L);
    m.ising->getUMPO(evol, delta, 0., true, 2);
    vector<double> energies;
    for (int cnt = 0; cnt < M; cnt++) {
      MPS aux(state);
      contractor.optimize(evol, aux, state, D);
      state.gaugeCond('R', true);
      energies.push_back(real(contractor.contract(state, m.H(), state)));
    }
    print_json({{"steps", (double)M}}, {{"energies", energies}});
  } else if (cmd == "evolve") {
    Model m = make_model(argv[2]);
    int D = atoi(argv[3]);
    int M = atoi(argv[4]);
    double dt = atof(argv[5]);
    contractor.setConvTol(atof(argv[6]));
    MPS state;
    state.importMPS(argv[7]);
    int L = m.L;
    MPO evol(L);
    m.ising->getUMPO(evol, dt, 0., false, 2);
    vector<double> sx_center, energies, entropies;
    mwArray sx = pauli("sx");
    for (int cnt = 0; cnt < M; cnt++) {
      MPS aux(state);
      contractor.optimize(evol, aux, state, D);
      vector<double> ex = expectations(state, sx);
      sx_center.push_back(ex[L / 2]);
      state.gaugeCond('L', 1);
      energies.push_back(real(contractor.contract(state, m.H(), state)));
      entropies.push_back(contractor.getEntropy(state, L / 2));
    }
    state.exportMPS(argv[8]);
    print_json({{"steps", (double)M}},
               {{"sx_center", sx_center}, {"energies", energies}, {"entropy_center", entropies}});
  } else if (cmd == "expect") {
    MPS s;
    s.importMPS(argv[2]);
    vector<double> ex = expectations(s, pauli(argv[3]));
    print_json({{"L", (double)s.getLength()}}, {{"values", ex}});
  } else if (cmd == "entropy") {
    MPS s;
    s.importMPS(argv[2]);
    double S = contractor.getEntropy(s, atoi(argv[3]));
    print_json({{"S", S}});
  } else if (cmd == "schmidt") {
    MPS s;
    s.importMPS(argv[2]);
    vector<complex_t> lam;
    contractor.getSchmidtValues(s, lam, atoi(argv[3]));
    vector<double> re;
    for (auto& c : lam) re.push_back(c.re);
    print_json({{"n", (double)re.size()}}, {{"values", re}});
  } else if (cmd == "truncate") {
    MPS s;
    s.importMPS(argv[2]);
    MPS t(s, atoi(argv[3]));
    t.exportMPS(argv[4]);
    print_json({{"bond", (double)t.getBond()}, {"normfact", t.getNormFact()}});
  } else if (cmd == "applympo") {
    Model m = make_model(argv[2]);
    MPO U(m.L);
    m.ising->getUMPO(U, atof(argv[3]), 0., atoi(argv[4]) != 0, 2);
    const int D = atoi(argv[5]);
    const bool dagger = atoi(argv[6]) != 0;
    const char dir = argv[7][0];
    MPS s;
    s.importMPS(argv[8]);
    MPS t(s);
    if (D > 0) t.approximate(U, s, D, dagger ? 'U' : 'D', dir);
    else t.applyExactly(U, dagger, dir);
    t.exportMPS(argv[9]);
    print_json({{"bond", (double)t.getBond()}, {"normfact", t.getNormFact()}});
  } else if (cmd == "savempo") {
    Model m = make_model(argv[2]);
    m.H().saveMPO(argv[3]);
    print_json({{"L", (double)m.L}});
  } else if (cmd == "optsum") {
    int D = atoi(argv[2]);
    contractor.setConvTol(atof(argv[3]));
    MPS init;
    init.importMPS(argv[4]);
    vector<MPS*> own;
    vector<const MPS*> kets;
    vector<complex_t> beta;
    for (int a = 6; a + 2 < argc; a += 3) {
      MPS* k = new MPS();
      k->importMPS(argv[a]);
      own.push_back(k);
      kets.push_back(k);
      beta.push_back((complex_t){atof(argv[a + 1]), atof(argv[a + 2])});
    }
    contractor.optimizeSum(kets, beta, init, D);
    init.exportMPS(argv[5]);
    print_json({{"normfact", init.getNormFact()}, {"terms", (double)kets.size()}});
    for (auto* k : own) delete k;
  } else if (cmd == "gauge") {
    MPS s;
    s.importMPS(argv[2]);
    s.gaugeCond(argv[3][0], true);
    s.exportMPS(argv[4]);
    print_json({{"bond", (double)s.getBond()}});
  } else if (cmd == "profile") {
    // Bounded sample of the ground-state sweep: the reference's own site
    // step (environment updates, TensorMultiplierOffset + eigensolver, QR
    // gauge move) on `nsites` consecutive sites around the chain centre.
    // Reports wall time and algorithmic flops (same formulas as the GPU
    // counters) so the caller can scale to a full solve.
    Model m = make_model(argv[2]);
    int D = atoi(argv[3]);
    contractor.setEigTol(atof(argv[4]));
    MPS st;
    st.importMPS(argv[5]);
    int nsites = atoi(argv[6]);
    const MPO& H = m.H();
    int L = m.L;
    st.gaugeCond('R', 1);
    st.gaugeCond('L', 1);
    auto mvflops = [&](int d, int w1, int w2, int dl, int dr) {
      return 8.0 * ((double)dl * w1 * dl * d * dr + (double)dl * d * d * w1 * w2 * dr + (double)dl * d * dr * w2 * dr);
    };
    int pos0 = argc > 7 ? atoi(argv[7]) : max(1, L / 2 - nsites / 2);
    pos0 = max(0, min(pos0, L - 2));
    vector<mwArray> Ls(L), Rs(L);
    Ls[0] = mwArray(ONE_c); Ls[0].reshape(Indices(1, 1, 1));
    Rs[L - 1] = mwArray(ONE_c); Rs[L - 1].reshape(Indices(1, 1, 1));
    for (int k = L - 2; k >= pos0; k--)
      H.getOp(k + 1).contractR(Rs[k], Rs[k + 1], st.getA(k + 1), st.getA(k + 1));
    for (int k = 1; k <= pos0; k++)
      H.getOp(k - 1).contractL(Ls[k], Ls[k - 1], st.getA(k - 1), st.getA(k - 1));
    struct timespec t0, t1;
    clock_gettime(CLOCK_MONOTONIC, &t0);
    double flops = 0.0;
    long long iters = 0;
    for (int pos = pos0; pos < pos0 + nsites && pos < L - 1; pos++) {
      const Site& A = st.getA(pos);
      int d = A.getd(), dl = A.getDl(), dr = A.getDr();
      const mwArray& W = H.getOp(pos).getFullData();
      int w1 = W.getDimension(1), w2 = W.getDimension(3);
      TensorMultiplierOffset multi(Ls[pos], W, Rs[pos], 0.);
      vector<complex_t> vals;
      mwArray U(A.getA());
      U.reshape(Indices(-1, 1));
      // count products through the eigensolver (one per Lanczos iteration)
      struct Counting : public Multiplier {
        Multiplier& in; long long n = 0;
        Counting(Multiplier& m_) : in(m_) {}
        void product(const mwArray& x, mwArray& y) { n++; in.product(x, y); }
        int getSize() const { return in.getSize(); }
        void getFullTensor(mwArray& r) { in.getFullTensor(r); }
      } cm(multi);
      wrapper::eigs_primme(cm, 1, primme_smallest, vals, U, 0.);
      iters += cm.n;
      flops += cm.n * mvflops(d, w1, w2, dl, dr);
      U.resize(Indices(U.getDimension(0), 1));
      st.setA(pos, U);
      st.gaugeCond(pos, 'R', true);
      int K = min(d * dl, dr);
      flops += 8.0 * 2.0 * (2.0 * d * dl * dr * K - (d * dl + dr) * (double)K * K + 2.0 * K * K * K / 3.0);
      H.getOp(pos).contractL(Ls[pos + 1], Ls[pos], st.getA(pos), st.getA(pos));
      flops += mvflops(d, w1, w2, dl, st.getA(pos).getDr());
    }
    clock_gettime(CLOCK_MONOTONIC, &t1);
    double secs = (t1.tv_sec - t0.tv_sec) + 1e-9 * (t1.tv_nsec - t0.tv_nsec);
    print_json({{"seconds", secs}, {"flops", flops}, {"iterations", (double)iters},
                {"pos0", (double)pos0}, {"nsites", (double)min(nsites, L - 1 - pos0)}});
  } else {
    cerr << "unknown command " << cmd << endl;
    return 2;
  }
  return 0;
}
