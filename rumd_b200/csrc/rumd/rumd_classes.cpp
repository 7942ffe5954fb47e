// Implementation of the RUMD class surface over the rumd_b200 C ABI.
#include "rumd_classes.h"

#include <zlib.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <iomanip>
#include <iostream>
#include <sstream>

#include "rumd_b200.h"

namespace rumd {

namespace {
constexpr int kNumParam = 12;  // NumParam, rumd_base.h

std::vector<std::string> split(const std::string& s, char sep) {
  std::vector<std::string> out;
  std::string cur;
  std::istringstream is(s);
  while (std::getline(is, cur, sep)) out.push_back(cur);
  return out;
}

// "Class,p1,p2,..." -> class name and the parameters as floats (the format
// of RUMD's info strings, ParseInfoString.cc:6-34).
std::string parse_info(const std::string& info, std::vector<float>& params) {
  params.clear();
  std::vector<std::string> parts = split(info, ',');
  if (parts.empty()) return "";
  for (size_t k = 1; k < parts.size(); ++k) {
    if (parts[k].empty()) continue;
    char* end = nullptr;
    const float v = std::strtof(parts[k].c_str(), &end);
    if (end == parts[k].c_str()) throw RUMD_Error("[None]", "ParseInfoString", "Failed to read parameter from infoStr " + info);
    params.push_back(v);
  }
  return parts[0];
}
}  // namespace

// ---------------------------------------------------------------------------
// NeighborList
// ---------------------------------------------------------------------------

void NeighborList::SetNB_Method(const std::string& m) {
  if (m != "default" && m != "sort" && m != "n2")
    throw RUMD_Error("NeighborList", "SetNB_Method", std::string("Unrecognized NB_method: ") + m);
  method = m;
}

int NeighborList::MethodCode() const {
  if (method == "sort") return 0;
  if (method == "n2") return 1;
  return -1;
}

// ---------------------------------------------------------------------------
// PairPotential family
// ---------------------------------------------------------------------------

float Pot_IPL_12_6::ComputeInteraction_CPU(float dist2, const float* param, float* u) const {
  // Pot_IPL_12_6::ComputeInteraction on the host, float arithmetic
  // (PairPotential.h:161-168), used for the shift constants
  volatile float invDist2 = 1.0f / dist2;
  volatile float invDist6 = invDist2 * invDist2 * invDist2;
  volatile float temp = param[1] * invDist6;
  volatile float t2 = 12.f * temp;
  volatile float t3 = 6.f * param[2];
  volatile float s = invDist6 * invDist2 * (t2 + t3);
  volatile float uu = invDist6 * (temp + param[2]);
  *u += uu;
  return s;
}

void PairPotential::StoreParams(unsigned i, unsigned j, std::vector<float> p) {
  if (p.size() + 2 > (size_t)kNumParam)
    throw RUMD_Error(GetID_String(), "CopyParamsToGPU", "RUMD requires more allocated parameters to run");
  p.resize(kNumParam, 0.f);
  float u = 0.f, s = 0.f;
  const float Rcut = p[0];
  if (Rcut > 0.0f) s = ComputeInteraction_CPU(Rcut * Rcut, p.data(), &u);
  p[kNumParam - 1] = u;
  p[kNumParam - 2] = s * Rcut;
  params_map[{i, j}] = p;
  if (i != j && assume_Newton3) params_map[{j, i}] = p;
  ParamsChanged();
}

void PairPotential::ParamsChanged() {
  if (sample) sample->PotentialChanged();
}

void Pot_IPL_12_6::SetParams(unsigned i, unsigned j, float A12, float A6, float Rcut) {
  StoreParams(i, j, {Rcut, A12, A6});
}

void Pot_LJ_12_6::SetParams(unsigned i, unsigned j, float Sigma, float Epsilon, float Rcut) {
  // Pot_LJ_12_6::SetParams (PairPotential.h:202-207): coefficients in double,
  // stored as float; cut-off in units of sigma
  Pot_IPL_12_6::SetParams(i, j, (float)(4. * Epsilon * std::pow((double)Sigma, 12.)),
                          (float)(-4. * Epsilon * std::pow((double)Sigma, 6.)), Rcut * Sigma);
}

void Pot_LJ_12_6_smooth_2_4::SetParams(unsigned i, unsigned j, float Sigma, float Epsilon, float Rcut) {
  // Pot_LJ_12_6_smooth_2_4::SetParams (PairPotential.h:232-246): c2, c4 in
  // double from Rcut in units of sigma, stored as float
  const float c2 = (float)(48. * std::pow((double)Rcut, -14.0) - 15. * std::pow((double)Rcut, -8.));
  const float c4 = (float)(6. * std::pow((double)Rcut, -10.0) - 21. * std::pow((double)Rcut, -16.));
  StoreParams(i, j, {Rcut * Sigma, 1.0f / (Sigma * Sigma), 4.0f * Epsilon, c2, c4});
}

float Pot_LJ_12_6_smooth_2_4::ComputeInteraction_CPU(float dist2, const float* param, float* u) const {
  // Pot_LJ_12_6_smooth_2_4::ComputeInteraction on the host, float arithmetic
  // (PairPotential.h:248-255), used for the shift constants
  volatile float Dist2 = dist2 * param[1];
  volatile float invDist2 = 1.0f / Dist2;
  volatile float invDist6 = invDist2 * invDist2 * invDist2;
  volatile float a = invDist2 * invDist6;
  volatile float b = 12.f * invDist6 - 6.f;
  volatile float c = 2.0f * param[3];
  volatile float d = 4.0f * param[4] * Dist2;
  volatile float s = param[2] * param[1] * (a * b - c - d);
  volatile float e = invDist6 * (invDist6 - 1.0f);
  volatile float g = param[3] * Dist2;
  volatile float h = param[4] * Dist2 * Dist2;
  *u += param[2] * (e + g + h);
  return s;
}

Pot_IPL_n::Pot_IPL_n(float n_, CutoffMethod m) : PairPotential(m), n(n_) {
  std::ostringstream ss;
  ss << "potIPL_" << n_;
  SetID_String(ss.str());
}

void Pot_IPL_n::SetParams(unsigned i, unsigned j, float Sigma, float Epsilon, float Rcut) {
  // Pot_IPL_n::SetParams (PairPotential.h:616-628)
  StoreParams(i, j, {Rcut * Sigma, 1.f / (Sigma * Sigma), Epsilon, n});
}

float Pot_IPL_n::ComputeInteraction_CPU(float dist2, const float* param, float* u) const {
  // Pot_IPL_n::ComputeInteraction on the host (PairPotential.h:630-636)
  volatile float invDist2 = 1.0f / (dist2 * param[1]);
  volatile float invDist_n = std::exp(std::log(invDist2) * param[3] * 0.5f);
  volatile float s = param[1] * param[2] * param[3] * invDist_n * invDist2;
  *u += param[2] * invDist_n;
  return s;
}

float PairPotential::GetPotentialParameter(unsigned t1, unsigned t2, unsigned k) const {
  auto it = params_map.find({t1, t2});
  if (it == params_map.end() || k >= it->second.size()) return 0.f;
  return it->second[k];
}

std::vector<float> PairPotential::GetPotentialParameters(unsigned num_types) const {
  std::vector<float> v;
  for (unsigned i = 0; i < num_types; ++i)
    for (unsigned j = 0; j < num_types; ++j)
      for (unsigned p = 0; p < (unsigned)kNumParam - 2; ++p) v.push_back(GetPotentialParameter(i, j, p));
  return v;
}

std::vector<float> PairPotential::ParamTable(unsigned T) const {
  std::vector<float> t((size_t)T * T * kNumParam, 0.f);
  for (const auto& kv : params_map) {
    unsigned i = kv.first.first, j = kv.first.second;
    if (i >= T || j >= T) continue;
    std::copy(kv.second.begin(), kv.second.end(), t.begin() + ((size_t)i * T + j) * kNumParam);
  }
  return t;
}

float PairPotential::GetMaxCutoff() const {
  float m = 0.f;
  for (const auto& kv : params_map) m = std::max(m, kv.second[0]);
  return m;
}

void PairPotential::SetNbListSkin(float s) {
  neighborList.SetSkin(s);
  ParamsChanged();
}

void PairPotential::SetNB_Method(const std::string& m) {
  neighborList.SetNB_Method(m);
  if (sample && sample->HasReplica()) {
    int rc = b2md_replica_set_nb_method(sample->Engine(), sample->ReplicaId(), neighborList.MethodCode());
    if (rc) throw RUMD_Error("NeighborList", "SetNB_Method", b2md_last_error());
  }
}

unsigned PairPotential::GetActualMaxNumNbrs() const {
  if (!sample || !sample->HasReplica()) return 0;
  return (unsigned)sample->Stats()[B2MD_STAT_ACTUAL_MAX_NBRS];
}

void PairPotential::CalcF(bool /*initialize*/, bool calc_stresses) {
  if (!sample) throw RUMD_Error(GetID_String(), "CalcF", "potential has no sample");
  sample->CalcF(calc_stresses);
}

double PairPotential::GetPotentialEnergy() {
  if (!sample) throw RUMD_Error(GetID_String(), "GetPotentialEnergy", "potential has no sample");
  return sample->GetPotentialEnergy();
}

// ---------------------------------------------------------------------------
// Integrators
// ---------------------------------------------------------------------------

void Integrator::SetTimeStep(float dt) {
  if (!(dt > 0.f)) throw RUMD_Error("Integrator", "SetTimeStep", "time step must be positive");
  timeStep = dt;
}

IntegratorNVT::IntegratorNVT(float dt) {
  timeStep = dt;
  thermostatOn = 0u;
  id = "IntegratorNVT";
}

IntegratorNVT::IntegratorNVT(float dt, double T, double tau) {
  timeStep = dt;
  targetTemperature = T;
  thermostatRelaxationTime = tau;
  thermostatOn = ~0u;
  id = "IntegratorNVT";
}

void IntegratorNVT::PushSettings() {
  if (!sample || !sample->HasReplica()) return;
  int rc = b2md_replica_set_integrator(sample->Engine(), sample->ReplicaId(), timeStep, targetTemperature,
                                       thermostatRelaxationTime, temperatureChangePerTimeStep, thermostatOn);
  if (rc) throw RUMD_Error("IntegratorNVT", "PushSettings", b2md_last_error());
}

void IntegratorNVT::SetTimeStep(float dt) {
  Integrator::SetTimeStep(dt);
  PushSettings();
}

std::string IntegratorNVT::GetInfoString(unsigned precision) const {
  std::ostringstream o;
  o << std::setprecision((int)precision);
  if (thermostatOn)
    o << "IntegratorNVT," << GetTimeStep() << "," << GetTargetTemperature() << "," << GetRelaxationTime() << ","
      << GetThermostatState();
  else
    o << "IntegratorNVE," << GetTimeStep();
  return o.str();
}

void IntegratorNVT::InitializeFromInfoString(const std::string& infoStr, bool verbose) {
  std::vector<float> p;
  const std::string cls = parse_info(infoStr, p);
  const bool nvt = cls == "IntegratorNVT";
  if (!nvt && cls != "IntegratorNVE")
    throw RUMD_Error("IntegratorNVT", "InitializeFromInfoString", "Expected IntegratorNVT or IntegratorNVE");
  if (p.size() != (nvt ? 4u : 1u))
    throw RUMD_Error("IntegratorNVT", "InitializeFromInfoString", "Wrong number of parameters in infoStr");
  if (verbose) std::cout << "[Info] Initializing " << cls << ". time step:" << p[0] << std::endl;
  SetTimeStep(p[0]);
  if (nvt) {
    SetTargetTemperature(p[1]);
    SetRelaxationTime(p[2]);
    SetThermostatState(p[3]);
  }
}

void IntegratorNVT::SetRelaxationTime(float tau) {
  thermostatRelaxationTime = tau;
  SetThermostatState(0.0);  // IntegratorNVT.cu:132-135
  PushSettings();
}

void IntegratorNVT::SetTargetTemperature(double T, bool reset) {
  targetTemperature = T;
  PushSettings();
  if (reset) SetThermostatState(0.0);
}

void IntegratorNVT::SetThermostatState(double Ps) {
  xi0 = Ps;
  if (sample && sample->HasReplica()) {
    int rc = b2md_replica_set_xi(sample->Engine(), sample->ReplicaId(), Ps);
    if (rc) throw RUMD_Error("IntegratorNVT", "SetThermostatState", b2md_last_error());
  }
}

void IntegratorNVT::SetThermostatOn(bool on) {
  thermostatOn = on ? ~0u : 0u;
  PushSettings();
}

void IntegratorNVT::SetThermostatOnParticleType(unsigned type, bool on) {
  if (type > 31) throw RUMD_Error("IntegratorNVT", "SetThermostatOnParticleType", "The particle type number is larger than 31");
  if (on) thermostatOn |= (1u << type);
  else thermostatOn &= ~(1u << type);
  PushSettings();
}

void IntegratorNVT::SetTemperatureChangePerTimeStep(double dT) {
  temperatureChangePerTimeStep = dT;
  PushSettings();
}

double IntegratorNVT::GetTargetTemperature() const {
  if (sample && sample->HasReplica()) return sample->Stats()[B2MD_STAT_TARGET_T];
  return targetTemperature;
}

double IntegratorNVT::GetThermostatState() const {
  if (!thermostatOn) return 0.0;
  if (sample && sample->HasReplica()) return sample->Stats()[B2MD_STAT_XI];
  return xi0;
}

void IntegratorNVT::Integrate() {
  if (!sample) throw RUMD_Error("IntegratorNVT", "Integrate", "Sample has not been set");
  sample->EnsureReplica();
  int rc = b2md_integrate(sample->Engine());
  if (rc) throw RUMD_Error("IntegratorNVT", "Integrate", b2md_last_error());
}

double IntegratorNVT::GetKineticEnergy(bool /*copy*/) const {
  // IntegratorNVT::GetKineticEnergy (IntegratorNVT.cu:316-356): leap-frog
  // average of m v^2 at t - h/2 and t + h/2, the latter from the current forces
  if (!sample) throw RUMD_Error("IntegratorNVT", "GetKineticEnergy", "Sample has no particles");
  std::vector<float> v = sample->GetField(B2MD_FIELD_VEL);
  std::vector<float> f = sample->GetField(B2MD_FIELD_FORCE);
  std::vector<float> r = sample->GetField(B2MD_FIELD_POS);
  double xi = GetThermostatState();
  double ke = 0.0;
  const size_t n = sample->GetNumberOfParticles();
  for (size_t i = 0; i < n; ++i) {
    float invm = v[4 * i + 3];
    double mass = 1.f / invm;
    float hm = invm * timeStep;
    int t;
    std::memcpy(&t, &r[4 * i + 3], 4);
    bool on = (thermostatOn >> t) & 1u;
    float factor = on ? 0.5f * timeStep * (float)xi : 0.f;
    float plus = 1.f / (1.f + factor), minus = 1.f - factor;
    float vf[3];
    double vb = 0, vv = 0;
    for (int d = 0; d < 3; ++d) {
      vf[d] = plus * (minus * v[4 * i + d] + hm * f[4 * i + d]);
      vb += (double)v[4 * i + d] * v[4 * i + d];
      vv += (double)vf[d] * vf[d];
    }
    ke += mass * ((vb + vv) / 2.0);
  }
  return 0.5 * ke;
}

void IntegratorNVT::SetMomentumToZero() {
  if (!sample) throw RUMD_Error("IntegratorNVT", "SetMomentumToZero", "Sample has not been set");
  sample->EnsureReplica();
  int rc = b2md_zero_momentum(sample->Engine());
  if (rc) throw RUMD_Error("IntegratorNVT", "SetMomentumToZero", b2md_last_error());
}

// ---------------------------------------------------------------------------
// Sample
// ---------------------------------------------------------------------------

Sample::Sample(unsigned pb_, unsigned tp_) : pb(pb_), tp(tp_), user_pb(pb_), user_tp(tp_) {}

Sample::~Sample() {
  if (eng) b2md_engine_destroy(eng);
}

void Sample::Check(int rc, const char* method) const {
  if (rc == B2MD_OK) return;
  if (rc == B2MD_ERR_ARG) throw RUMD_cudaResourceError("Sample", method, b2md_last_error());
  throw RUMD_Error("Sample", method, b2md_last_error());
}

void Sample::ChooseLaunch() {
  // Defaults by size, as Sample(pb=0, tp=0) does (Sample.cu:208-215), with
  // B200 shapes: tp = 4 threads per particle, 64 particles per block.
  unsigned n = GetNumberOfParticles();
  // RUMD's shapes (pb 16..192, tp up to 64) are accepted; the engine maps
  // them onto whole-warp tiles and tp in {1, 2, 4, 8} (b2md_engine_set_launch)
  // and GetParticlesPerBlock / GetThreadsPerParticle report what it runs.
  pb = user_pb ? user_pb : (n > 10000 ? 64 : 32);
  tp = user_tp ? user_tp : 4;
  if (pb < 1 || pb > 1024 || tp < 1 || tp > 64)
    throw RUMD_cudaResourceError("Sample", "SetPB_TP", "pb must be 1..1024 and tp 1..64");
}

void Sample::SyncLaunch() {
  int p = 0, t = 0;
  Check(b2md_engine_get_launch(eng, &p, &t), "GetKernelPlan");
  pb = (unsigned)p;
  tp = (unsigned)t;
}

void Sample::SetPB_TP(unsigned pb_, unsigned tp_) {
  user_pb = pb_;
  user_tp = tp_;
  ChooseLaunch();
  if (eng) {
    Check(b2md_engine_set_launch(eng, (int)pb, (int)tp), "SetPB_TP");
    SyncLaunch();
  }
}

void Sample::SetConfiguration(const std::vector<float>& pos3, const std::vector<int>& types,
                              const std::vector<float>& box_, const std::vector<float>& masses_per_type,
                              const std::vector<float>& vel3, const std::vector<int>& images3) {
  size_t n = types.size();
  if (n < 2 || pos3.size() != 3 * n) throw RUMD_Error("Sample", "SetConfiguration", "need 3 coordinates per particle");
  if (box_.size() != 3) throw RUMD_Error("Sample", "SetConfiguration", "box needs 3 lengths");
  int maxt = 0;
  for (int t : types) {
    if (t < 0) throw RUMD_Error("Sample", "SetConfiguration", "negative particle type");
    maxt = std::max(maxt, t);
  }
  Invalidate();
  box = box_;
  mass = masses_per_type;
  if ((int)mass.size() < maxt + 1) mass.resize(maxt + 1, 1.f);
  type = types;
  pos.assign(4 * n, 0.f);
  vel.assign(4 * n, 0.f);
  im.assign(3 * n, 0);
  for (size_t i = 0; i < n; ++i) {
    for (int d = 0; d < 3; ++d) {
      pos[4 * i + d] = pos3[3 * i + d];
      if (vel3.size() == 3 * n) vel[4 * i + d] = vel3[3 * i + d];
      if (images3.size() == 3 * n) im[3 * i + d] = images3[3 * i + d];
    }
    std::memcpy(&pos[4 * i + 3], &type[i], 4);
    vel[4 * i + 3] = 1.f / mass[type[i]];
  }
  ChooseLaunch();
}

unsigned Sample::GetNumberThisType(unsigned t) const {
  return (unsigned)std::count(type.begin(), type.end(), (int)t);
}

float Sample::GetMass(unsigned t) const {
  if (t >= mass.size()) throw RUMD_Error("ParticleData", "GetMass", "Type index too large");
  return mass[t];
}

void Sample::SetMass(unsigned t, float m) {
  if (t >= mass.size()) throw RUMD_Error("ParticleData", "SetMass", "Type index too large");
  if (!(m > 0.f)) throw RUMD_Error("ParticleData", "SetMass", "mass must be positive");
  std::vector<float> v = GetField(B2MD_FIELD_VEL);
  mass[t] = m;
  for (size_t i = 0; i < type.size(); ++i)
    if (type[i] == (int)t) v[4 * i + 3] = 1.f / m;
  vel = v;
  if (HasReplica()) Check(b2md_replica_set(eng, rid, B2MD_FIELD_VEL, v.data()), "SetMass");
}

// Sample::SetPotential (Sample.cu:251-259): the potential list becomes this
// one potential.
void Sample::SetPotential(Potential* p) {
  auto* pp = dynamic_cast<PairPotential*>(p);
  if (!pp) throw RUMD_Error("Sample", "SetPotential", "only Lennard-Jones pair potentials are supported");
  if (pot && pot != pp) pot->SetSample(nullptr);
  if (pot2 && pot2 != pp) pot2->SetSample(nullptr);
  pot2 = nullptr;
  pot = pp;
  pot->SetSample(this);
  PotentialChanged();
}

// Sample::AddPotential (Sample.cu:261-278): one more potential in the list
// that CalcF evaluates, the first storing forces, energies, virials and
// stresses and the other adding to them (Sample.cu:335-336,
// PairPotential.cu:370-388).  The engine holds two pair potentials per
// sample, over one neighbour list built with the larger cut-off and the
// first potential's skin.
void Sample::AddPotential(Potential* p) {
  auto* pp = dynamic_cast<PairPotential*>(p);
  if (!pp) throw RUMD_Error("Sample", "AddPotential", "only Lennard-Jones pair potentials are supported");
  if (!pot) {
    SetPotential(p);
    return;
  }
  if (pp == pot || pp == pot2) throw RUMD_Error("Sample", "AddPotential", "this potential is already in the list");
  if (pot2) throw RUMD_Error("Sample", "AddPotential", "at most two pair potentials per sample are supported");
  pot2 = pp;
  pot2->SetSample(this);
  PotentialChanged();
}

std::vector<PairPotential*> Sample::GetPotentials() const {
  std::vector<PairPotential*> out;
  if (pot) out.push_back(pot);
  if (pot2) out.push_back(pot2);
  return out;
}

void Sample::SetIntegrator(Integrator* i) {
  itg = i;
  if (itg) itg->SetSample(this);
  IntegratorChanged();
}

void Sample::Invalidate() {
  if (eng && rid >= 0) b2md_replica_remove(eng, rid);
  rid = -1;
}

void Sample::EnsureReplica() {
  if (rid >= 0) return;
  if (type.empty()) throw RUMD_Error("Sample", "CalcF", "No configuration has been read");
  if (!pot) throw RUMD_Error("Sample", "CalcF", "No potential has been set");
  ChooseLaunch();
  if (!eng) {
    Check(b2md_engine_create(0, (long long)type.size(), 1, 0, (int)pb, (int)tp, &eng), "Sample");
    SyncLaunch();
  }
  std::vector<float> table = pot->ParamTable(GetNumberOfTypes());
  b2md_replica_desc d;
  std::memset(&d, 0, sizeof(d));
  d.n = (int)type.size();
  d.ntypes = (int)GetNumberOfTypes();
  for (int k = 0; k < 3; ++k) d.box[k] = box[k];
  d.params = table.data();
  d.cutoff_method = pot->GetCutoffMethod();
  d.skin = pot->GetNbListSkin();
  auto* nvt = dynamic_cast<IntegratorNVT*>(itg);
  d.dt = itg ? itg->GetTimeStep() : (file_dt > 0.f ? file_dt : 0.005f);
  d.target_T = nvt ? nvt->GetTargetTemperature() : 0.0;
  d.tau = nvt ? nvt->GetRelaxationTime() : 0.2;
  if (!(d.tau > 0.0)) d.tau = 0.2;
  d.dT_per_step = nvt ? nvt->GetTemperatureChangePerTimeStep() : 0.0;
  d.xi = nvt ? nvt->initialXi() : file_xi;
  d.thermostat_mask = nvt ? nvt->GetThermostatMask() : 0u;
  d.reset_interval = 0;
  d.max_nbrs = (int)pot->GetNeighborList().GetMaxNumNbrs();
  d.potential = pot->PotentialKind();
  Check(b2md_replica_add(eng, &d, pos.data(), vel.data(), im.data(), &rid), "SetNumberOfParticles");
  if (pot2) {
    std::vector<float> t2 = pot2->ParamTable(GetNumberOfTypes());
    Check(b2md_replica_add_potential(eng, rid, (int)GetNumberOfTypes(), t2.data(), pot2->GetCutoffMethod(),
                                     pot2->PotentialKind()),
          "AddPotential");
  }
  int m = pot->GetNeighborList().MethodCode();
  if (m != -1) Check(b2md_replica_set_nb_method(eng, rid, m), "SetNB_Method");
  if (elog_interval > 0) Check(b2md_replica_set_energy_log(eng, rid, elog_interval, elog_capacity), "SetEnergyLog");
}

void Sample::SetEnergyLog(int interval, int capacity) {
  elog_interval = interval;
  elog_capacity = capacity;
  if (HasReplica()) Check(b2md_replica_set_energy_log(eng, rid, interval, capacity), "SetEnergyLog");
}

std::vector<double> Sample::GetEnergyLog() const {
  if (!HasReplica() || elog_capacity <= 0) return {};
  std::vector<double> out((size_t)elog_capacity * 5);
  int cnt = 0;
  Check(b2md_replica_energy_log(eng, rid, out.data(), elog_capacity, &cnt), "GetEnergyLog");
  out.resize((size_t)cnt * 5);
  return out;
}

void Sample::PotentialChanged() {
  if (!HasReplica() || !pot) return;
  std::vector<float> table = pot->ParamTable(GetNumberOfTypes());
  Check(b2md_replica_set_potential(eng, rid, (int)GetNumberOfTypes(), table.data(), pot->GetCutoffMethod(),
                                   pot->GetNbListSkin(), pot->PotentialKind()),
        "SetPotential");
  if (pot2) {
    std::vector<float> t2 = pot2->ParamTable(GetNumberOfTypes());
    Check(b2md_replica_add_potential(eng, rid, (int)GetNumberOfTypes(), t2.data(), pot2->GetCutoffMethod(),
                                     pot2->PotentialKind()),
          "AddPotential");
  }
}

void Sample::IntegratorChanged() {
  if (!HasReplica()) return;
  if (auto* nvt = dynamic_cast<IntegratorNVT*>(itg)) {
    nvt->PushSettings();
    nvt->SetThermostatState(nvt->initialXi());
  }
}

void Sample::CalcF(bool calc_stresses) {
  EnsureReplica();
  Check(b2md_calc_f(eng, calc_stresses ? 1 : 0), "CalcF");
}

void Sample::Run(long long nsteps, int reset_interval) {
  if (!itg) throw RUMD_Error("Sample", "Run", "Integrator has not been set");
  EnsureReplica();
  Check(b2md_replica_set_reset_interval(eng, rid, reset_interval), "Run");
  Check(b2md_run(eng, nsteps), "Run");
}

std::vector<double> Sample::Stats() const {
  std::vector<double> s(B2MD_NSTAT, 0.0);
  if (HasReplica()) Check(b2md_replica_stats(eng, rid, s.data()), "Stats");
  return s;
}

double Sample::GetPotentialEnergy(bool) const {
  if (!HasReplica()) throw RUMD_Error("Sample", "GetPotentialEnergy", "CalcF has not been called");
  return Stats()[B2MD_STAT_PE];
}

double Sample::GetVirial(bool) const {
  if (!HasReplica()) throw RUMD_Error("Sample", "GetVirial", "CalcF has not been called");
  return Stats()[B2MD_STAT_VIRIAL];
}

std::vector<double> Sample::GetStress(bool) const {
  if (!HasReplica()) throw RUMD_Error("Sample", "GetStress", "CalcF has not been called");
  std::vector<double> s(6);
  Check(b2md_replica_stress(eng, rid, include_kinetic_stress ? 1 : 0, s.data()), "GetStress");
  return s;
}

std::vector<float> Sample::GetField(int field) const {
  if (!HasReplica()) {
    if (field == B2MD_FIELD_POS) return pos;
    if (field == B2MD_FIELD_VEL) return vel;
    return std::vector<float>(4 * type.size(), 0.f);
  }
  std::vector<float> out(4 * type.size());
  Check(b2md_replica_get(eng, rid, field, out.data()), "GetField");
  return out;
}

std::vector<int> Sample::GetImages() const {
  if (!HasReplica()) return im;
  std::vector<int> out(3 * type.size());
  Check(b2md_replica_get(eng, rid, B2MD_FIELD_IMAGES, out.data()), "GetImages");
  return out;
}

void Sample::SetPositions(const std::vector<float>& pos3) {
  size_t n = type.size();
  if (pos3.size() != 3 * n) throw RUMD_Error("Sample", "SetPositions", "need 3 coordinates per particle");
  std::vector<float> p = GetField(B2MD_FIELD_POS);
  for (size_t i = 0; i < n; ++i)
    for (int d = 0; d < 3; ++d) p[4 * i + d] = pos3[3 * i + d];
  pos = p;
  if (HasReplica()) Check(b2md_replica_set(eng, rid, B2MD_FIELD_POS, p.data()), "SetPositions");
}

void Sample::SetVelocities(const std::vector<float>& vel3) {
  size_t n = type.size();
  if (vel3.size() != 3 * n) throw RUMD_Error("Sample", "SetVelocities", "need 3 components per particle");
  std::vector<float> v = GetField(B2MD_FIELD_VEL);
  for (size_t i = 0; i < n; ++i)
    for (int d = 0; d < 3; ++d) v[4 * i + d] = vel3[3 * i + d];
  vel = v;
  if (HasReplica()) Check(b2md_replica_set(eng, rid, B2MD_FIELD_VEL, v.data()), "SetVelocities");
}

void Sample::ExportNeighborList(std::vector<unsigned>& counts, std::vector<unsigned>& nbl, int max_nbrs) const {
  if (!HasReplica()) throw RUMD_Error("Sample", "ExportNeighborList", "CalcF has not been called");
  counts.assign(type.size(), 0);
  nbl.assign(type.size() * (size_t)max_nbrs, 0);
  Check(b2md_nbl_export(eng, rid, counts.data(), nbl.data(), max_nbrs), "ExportNeighborList");
}

std::vector<unsigned> Sample::ExportSortIndex() const {
  if (!HasReplica()) throw RUMD_Error("Sample", "ExportSortIndex", "CalcF has not been called");
  std::vector<unsigned> out(type.size());
  Check(b2md_sort_export(eng, rid, out.data()), "ExportSortIndex");
  return out;
}

// ---------------------------------------------------------------------------
// Configuration files (ConfigurationWriterReader.cu:90-343): gzip'd xyz with a
// key=value header line and a columns= list.
// ---------------------------------------------------------------------------

void Sample::ReadConf(const std::string& filename, bool init_itg) {
  gzFile fp = gzopen(filename.c_str(), "rb");
  if (!fp) throw RUMD_Error("Sample", "ReadConf", "cannot open " + filename);
  std::vector<char> buf(1 << 16);
  auto getline = [&](std::string& line) -> bool {
    line.clear();
    while (true) {
      if (!gzgets(fp, buf.data(), (int)buf.size())) return !line.empty();
      line += buf.data();
      if (!line.empty() && line.back() == '\n') {
        line.pop_back();
        return true;
      }
    }
  };
  auto fail = [&](const std::string& msg) {
    gzclose(fp);
    throw RUMD_Error("Sample", "ReadConf", msg);
  };
  std::string line;
  if (!getline(line)) fail("empty file");
  long n = std::strtol(line.c_str(), nullptr, 10);
  if (n < 2) fail("bad particle count");
  getline(line);
  std::map<std::string, std::string> meta;
  for (const std::string& tok : split(line, ' ')) {
    auto eq = tok.find('=');
    if (eq != std::string::npos) meta[tok.substr(0, eq)] = tok.substr(eq + 1);
  }
  // ConfigurationMetaData::ReadMetaData (ConfigurationMetaData.cc:166-214):
  // ioformat 1 carries dt, boxLengths and Nose-Hoover-Ps; ioformat 2 carries
  // integrator=Class,params and sim_box=Class,params
  if (!meta.count("ioformat")) fail("Did not find ioformat");
  const int iof = std::atoi(meta["ioformat"].c_str());
  if (iof != 1 && iof != 2) fail("ioformat must be 1 or 2");
  std::string box_info, itg_info;
  bool found_itg = false;
  file_xi = 0.0;
  file_dt = 0.f;
  if (iof == 1) {
    if (meta.count("boxLengths")) box_info = "RectangularSimulationBox," + meta["boxLengths"];
    if (meta.count("Nose-Hoover-Ps")) {
      file_xi = std::stod(meta["Nose-Hoover-Ps"]);
      found_itg = true;
    }
    if (meta.count("dt")) file_dt = std::stof(meta["dt"]);
  } else {
    if (meta.count("sim_box")) box_info = meta["sim_box"];
    if (meta.count("integrator")) {
      itg_info = meta["integrator"];
      found_itg = true;
      std::vector<float> ip;
      const std::string cls = parse_info(itg_info, ip);
      if (!ip.empty()) file_dt = ip[0];  // ConfigurationMetaData.cc:209-212
      if (cls == "IntegratorNVT" && ip.size() == 4) file_xi = ip[3];
    }
  }
  if (box_info.empty()) fail("Did not find box information");
  std::vector<float> L;
  if (parse_info(box_info, L) != "RectangularSimulationBox")
    fail("only RectangularSimulationBox is supported (file has " + box_info.substr(0, box_info.find(',')) + ")");
  if (L.size() == 1) L.assign(3, L[0]);
  if (L.size() != 3) fail("RectangularSimulationBox needs 3 lengths");
  if (!meta.count("columns")) fail("header needs columns=");
  file_ioformat = iof;
  file_integrator = itg_info;
  std::vector<std::string> cols = split(meta["columns"], ',');
  std::vector<float> masses;
  if (meta.count("mass"))
    for (auto& s : split(meta["mass"], ',')) masses.push_back(std::stof(s));
  if (meta.count("numTypes")) masses.resize(std::max<size_t>(masses.size(), std::stoul(meta["numTypes"])), 1.f);
  auto col = [&](const char* name) -> int {
    for (size_t k = 0; k < cols.size(); ++k)
      if (cols[k] == name) return (int)k;
    return -1;
  };
  int ct = col("type"), cx = col("x"), cy = col("y"), cz = col("z");
  int cvx = col("vx"), cvy = col("vy"), cvz = col("vz"), cix = col("imx"), ciy = col("imy"), ciz = col("imz");
  if (ct < 0 || cx < 0 || cy < 0 || cz < 0) fail("missing columns");
  std::vector<float> p3(3 * n), v3, i3f;
  std::vector<int> types(n), i3;
  if (cvx >= 0) v3.assign(3 * n, 0.f);
  if (cix >= 0) i3.assign(3 * n, 0);
  for (long i = 0; i < n; ++i) {
    if (!getline(line)) fail("file ends early");
    std::istringstream is(line);
    std::vector<double> v;
    double x;
    while (is >> x) v.push_back(x);
    if ((int)v.size() < (int)cols.size()) fail("short particle line");
    types[i] = (int)v[ct];
    p3[3 * i] = (float)v[cx]; p3[3 * i + 1] = (float)v[cy]; p3[3 * i + 2] = (float)v[cz];
    if (cvx >= 0) { v3[3 * i] = (float)v[cvx]; v3[3 * i + 1] = (float)v[cvy]; v3[3 * i + 2] = (float)v[cvz]; }
    if (cix >= 0) { i3[3 * i] = (int)v[cix]; i3[3 * i + 1] = (int)v[ciy]; i3[3 * i + 2] = (int)v[ciz]; }
  }
  gzclose(fp);
  SetConfiguration(p3, types, L, masses, v3, i3);
  // Sample::ReadConf(filename, init_itg) (Sample.cu:584-600)
  if (itg && init_itg && found_itg) {
    if (iof == 1) {
      if (auto* nvt = dynamic_cast<IntegratorNVT*>(itg)) nvt->SetThermostatState(file_xi);
    } else {
      itg->InitializeFromInfoString(itg_info);
    }
  }
}

void Sample::WriteConf(const std::string& filename) {
  std::vector<float> r = GetField(B2MD_FIELD_POS), v = GetField(B2MD_FIELD_VEL), f = GetField(B2MD_FIELD_FORCE),
                     w = GetField(B2MD_FIELD_VIRIAL);
  std::vector<int> imgs = GetImages();
  gzFile fp = gzopen(filename.c_str(), "wb");
  if (!fp) throw RUMD_Error("Sample", "WriteConf", "cannot open " + filename);
  // ConfigurationWriterReader::Write_ioformat2 (ConfigurationWriterReader.cu:90-141):
  // info strings with precision + 2 significant figures, the rest with
  // `precision` decimals (9, the restart writer's)
  const int precision = 9;
  std::ostringstream h;
  h << type.size() << "\nioformat=2 numTypes=" << mass.size();
  if (itg) h << " integrator=" << itg->GetInfoString(precision + 2);
  {
    std::ostringstream b;
    b << std::setprecision(precision + 2) << "RectangularSimulationBox," << box[0] << "," << box[1] << "," << box[2];
    h << " sim_box=" << b.str();
  }
  h << std::fixed << std::setprecision(precision) << " mass=";
  for (size_t t = 0; t < mass.size(); ++t) h << (t ? "," : "") << mass[t];
  h << " columns=type,x,y,z,imx,imy,imz,vx,vy,vz,fx,fy,fz,pe,vir\n";
  gzputs(fp, h.str().c_str());
  char line[512];
  for (size_t i = 0; i < type.size(); ++i) {
    snprintf(line, sizeof(line), "%d %.9f %.9f %.9f %d %d %d %.9f %.9f %.9f %.9f %.9f %.9f %.9f %.9f\n", type[i],
             r[4 * i], r[4 * i + 1], r[4 * i + 2], imgs[3 * i], imgs[3 * i + 1], imgs[3 * i + 2], v[4 * i],
             v[4 * i + 1], v[4 * i + 2], f[4 * i], f[4 * i + 1], f[4 * i + 2], f[4 * i + 3], w[4 * i + 3] / 2.0);
    gzputs(fp, line);
  }
  gzclose(fp);
}

}  // namespace rumd
