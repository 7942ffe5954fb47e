// RUMD's C++ object model for the LJ/NVT time step, re-implemented over the
// rumd_b200 C ABI (include/rumd_b200.h).
//
// The classes keep the reference's names, method names, argument meaning and
// error behaviour (RUMD_Error, include/rumd/RUMD_Error.h:10-31) so that code
// written against RUMD's Sample / PairPotential / Pot_LJ_12_6 / NeighborList /
// IntegratorNVT keeps working.  All numerical work happens in the engine on the
// GPU; these classes hold host-side settings and forward to the C ABI.
//
// Ownership follows the reference (Sample.h:33-90): a Sample holds non-owning
// pointers to its potential and integrator; the caller keeps them alive.
#pragma once
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

struct b2md_engine;

namespace rumd {

class RUMD_Error : public std::runtime_error {
 public:
  RUMD_Error(const std::string& cls, const std::string& method, const std::string& msg)
      : std::runtime_error(cls + "::" + method + ": " + msg), className(cls), methodName(method), errorStr(msg) {}
  std::string className, methodName, errorStr;
};

// Raised for launch-shape problems (RUMD_cudaResourceError, RUMD_Error.h:25-31).
class RUMD_cudaResourceError : public RUMD_Error {
 public:
  using RUMD_Error::RUMD_Error;
};

class Sample;

// NeighborList is a by-value member of PairPotential (PairPotential.h:46).
class NeighborList {
 public:
  NeighborList() = default;
  void SetSkin(float s) { skin = s; }
  float GetSkin() const { return skin; }
  // "default", "sort", "n2" (NeighborList.cu:226-245).  "none" is not provided.
  void SetNB_Method(const std::string& method);
  std::string GetNB_Method() const { return method; }
  void SetMaxNumNbrs(unsigned m) { max_nbrs = m; }
  unsigned GetMaxNumNbrs() const { return max_nbrs; }
  int MethodCode() const;

 private:
  float skin = 0.5f;  // NeighborList.cu:50
  std::string method = "default";
  unsigned max_nbrs = 0;
};

class Potential {
 public:
  virtual ~Potential() = default;
  virtual void SetSample(Sample* s) { sample = s; }
  virtual void CalcF(bool initialize, bool calc_stresses) = 0;
  virtual double GetPotentialEnergy() = 0;
  const std::string& GetID_String() const { return id; }
  void SetID_String(const std::string& s) { id = s; }
  void SetVerbose(bool v) { verbose = v; }
  bool IsMolecularPotential() const { return false; }
  bool EnergyIncludedInParticleSum() const { return true; }

 protected:
  Sample* sample = nullptr;
  std::string id = "potential";
  bool verbose = true;
};

class PairPotential : public Potential {
 public:
  enum CutoffMethod { NS = 0, SP = 1, SF = 2 };
  explicit PairPotential(CutoffMethod m) : cutoffMethod(m) { SetID_String("base_pair_pot"); }

  void CalcF(bool initialize, bool calc_stresses) override;
  double GetPotentialEnergy() override;

  // Parameter access (PairPotential.h:94-117).  NumParam-2 values per pair.
  float GetPotentialParameter(unsigned t1, unsigned t2, unsigned k) const;
  std::vector<float> GetPotentialParameters(unsigned num_types) const;
  // Full RUMD layout table (T*T*12) with the shift constants filled in
  // (PairPotential::CopyParamsToGPU, PairPotential.cu:82-125).
  std::vector<float> ParamTable(unsigned num_types) const;

  void SetNbListSkin(float s);
  float GetNbListSkin() const { return neighborList.GetSkin(); }
  void SetNB_Method(const std::string& m);
  std::string GetNB_Method() const { return neighborList.GetNB_Method(); }
  void SetNbMaxNumNbrs(unsigned m) { neighborList.SetMaxNumNbrs(m); }
  float GetMaxCutoff() const;
  int GetCutoffMethod() const { return cutoffMethod; }
  unsigned GetActualMaxNumNbrs() const;
  void SetAssumeNewton3(bool v) { assume_Newton3 = v; }
  // Which pair function the rows hold (B2MD_POT_*).
  virtual int PotentialKind() const { return 0; }
  NeighborList& GetNeighborList() { return neighborList; }
  const NeighborList& GetNeighborList() const { return neighborList; }

 protected:
  // Stores params (Rcut first) for pair (i, j) and, with Newton's third law,
  // for (j, i); recomputes the shift constants.
  void StoreParams(unsigned i, unsigned j, std::vector<float> p);
  virtual float ComputeInteraction_CPU(float dist2, const float* param, float* u) const = 0;
  void ParamsChanged();

  CutoffMethod cutoffMethod;
  std::map<std::pair<unsigned, unsigned>, std::vector<float>> params_map;
  NeighborList neighborList;
  bool assume_Newton3 = true;
};

// v(r) = A12/r^12 + A6/r^6 (PairPotential.h:135-169)
class Pot_IPL_12_6 : public PairPotential {
 public:
  explicit Pot_IPL_12_6(CutoffMethod m) : PairPotential(m) { SetID_String("potIPL_12_6"); }
  void SetParams(unsigned i, unsigned j, float A12, float A6, float Rcut);

 protected:
  float ComputeInteraction_CPU(float dist2, const float* param, float* u) const override;
};

// v(r) = 4 eps ((sigma/r)^12 - (sigma/r)^6) (PairPotential.h:186-208)
class Pot_LJ_12_6 : public Pot_IPL_12_6 {
 public:
  explicit Pot_LJ_12_6(CutoffMethod m) : Pot_IPL_12_6(m) { SetID_String("potLJ_12_6"); }
  void SetParams(unsigned i, unsigned j, float Sigma, float Epsilon, float Rcut);
};

// v(r) = 4 eps ((sigma/r)^12 - (sigma/r)^6 + c2 (r/sigma)^2 + c4 (r/sigma)^4),
// c2, c4 chosen so that the force and its derivative vanish at Rcut; the
// constant c0 that would make v(Rcut) = 0 is left to the ShiftedPotential
// cut-off (Pot_LJ_12_6_smooth_2_4, PairPotential.h:210-256).
class Pot_LJ_12_6_smooth_2_4 : public PairPotential {
 public:
  explicit Pot_LJ_12_6_smooth_2_4(CutoffMethod m) : PairPotential(m) { SetID_String("potLJ_12_6_smooth_2_4"); }
  void SetParams(unsigned i, unsigned j, float Sigma, float Epsilon, float Rcut);
  int PotentialKind() const override { return 1; }

 protected:
  float ComputeInteraction_CPU(float dist2, const float* param, float* u) const override;
};

// v(r) = eps (sigma/r)^n (Pot_IPL_n, PairPotential.h:603-637).
class Pot_IPL_n : public PairPotential {
 public:
  Pot_IPL_n(float n, CutoffMethod m);
  void SetParams(unsigned i, unsigned j, float Sigma, float Epsilon, float Rcut);
  int PotentialKind() const override { return 2; }
  float GetExponent() const { return n; }

 protected:
  float ComputeInteraction_CPU(float dist2, const float* param, float* u) const override;
  float n;
};

class Integrator {
 public:
  virtual ~Integrator() = default;
  virtual void SetSample(Sample* s) { sample = s; }
  virtual void Integrate() = 0;
  virtual double GetKineticEnergy(bool copy = true) const = 0;
  virtual void SetMomentumToZero() = 0;
  float GetTimeStep() const { return timeStep; }
  virtual void SetTimeStep(float dt);
  bool RequiresStress() const { return false; }
  const std::string& GetID_String() const { return id; }
  // "Class,p1,p2,..." as written to ioformat=2 files (IntegratorNVT.cu:252-290)
  virtual std::string GetInfoString(unsigned precision) const = 0;
  virtual void InitializeFromInfoString(const std::string& infoStr, bool verbose = false) = 0;

 protected:
  Sample* sample = nullptr;
  float timeStep = 0.f;
  std::string id = "integrator";
};

// Leap-frog NVE / Toxvaerd Nose-Hoover NVT (IntegratorNVT.h, IntegratorNVT.cu).
class IntegratorNVT : public Integrator {
 public:
  explicit IntegratorNVT(float timeStep);  // NVE
  IntegratorNVT(float timeStep, double targetTemperature, double thermostatRelaxationTime);

  void Integrate() override;
  double GetKineticEnergy(bool copy = true) const override;
  void SetMomentumToZero() override;
  void SetTimeStep(float dt) override;
  std::string GetInfoString(unsigned precision) const override;
  void InitializeFromInfoString(const std::string& infoStr, bool verbose = false) override;

  void SetRelaxationTime(float tau);
  void SetTargetTemperature(double T, bool reset = false);
  void SetThermostatState(double Ps);
  void SetThermostatOn(bool on = true);
  void SetThermostatOnParticleType(unsigned type, bool on);
  void SetTemperatureChangePerTimeStep(double dT);
  float GetRelaxationTime() const { return (float)thermostatRelaxationTime; }
  double GetTargetTemperature() const;
  double GetThermostatState() const;
  double GetTemperatureChangePerTimeStep() const { return temperatureChangePerTimeStep; }
  unsigned GetThermostatMask() const { return thermostatOn; }
  bool GetThermostatOn() const { return thermostatOn != 0; }
  // Settings pushed to the engine (called by Sample when the replica exists).
  void PushSettings();
  double initialXi() const { return xi0; }

 private:
  double targetTemperature = 0.0;
  double thermostatRelaxationTime = 0.2;
  double temperatureChangePerTimeStep = 0.0;
  unsigned thermostatOn = 0u;
  double xi0 = 0.0;
};

// IntegratorNVE is IntegratorNVT under another name (Swig/Integrators.i:16).
class IntegratorNVE : public IntegratorNVT {
 public:
  explicit IntegratorNVE(float timeStep) : IntegratorNVT(timeStep) { id = "IntegratorNVE"; }
};

class Sample {
 public:
  // Sample(pb, tp); 0 = choose by size (Sample.cu:36-39, 208-215).
  explicit Sample(unsigned pb = 0, unsigned tp = 0);
  ~Sample();
  Sample(const Sample&) = delete;
  Sample& operator=(const Sample&) = delete;

  // Configuration I/O (ConfigurationWriterReader.cu:90-343).
  // ConfigurationWriterReader::Read + ConfigurationMetaData::ReadMetaData
  // (Sample.cu:584-600, ConfigurationMetaData.cc:166-214): ioformat 1 or 2;
  // with init_itg the file's integrator state goes to the integrator.
  void ReadConf(const std::string& filename, bool init_itg = false);
  void WriteConf(const std::string& filename);
  // Direct configuration set-up (positions xyz, types, box, masses per type).
  void SetConfiguration(const std::vector<float>& pos3, const std::vector<int>& types, const std::vector<float>& box,
                        const std::vector<float>& masses_per_type, const std::vector<float>& vel3,
                        const std::vector<int>& images3);

  void SetPotential(Potential* p);
  void AddPotential(Potential* p);
  void SetIntegrator(Integrator* itg);
  Integrator* GetIntegrator() const { return itg; }
  PairPotential* GetPairPotential() const { return pot; }
  // the potentials CalcF evaluates (one or two)
  std::vector<PairPotential*> GetPotentials() const;

  void CalcF(bool calc_stresses = false);
  // Simulation.Run's time-step loop as fused device graphs (momentum reset
  // every reset_interval steps, then a final CalcF).
  void Run(long long nsteps, int reset_interval = 100);

  double GetPotentialEnergy(bool copy = true) const;
  double GetVirial(bool copy = true) const;
  std::vector<double> GetStress(bool copy = true) const;
  void SetIncludeKineticStress(bool v) { include_kinetic_stress = v; }

  unsigned GetNumberOfParticles() const { return (unsigned)type.size(); }
  unsigned GetNumberOfTypes() const { return (unsigned)mass.size(); }
  unsigned GetNumberThisType(unsigned t) const;
  float GetMass(unsigned t) const;
  void SetMass(unsigned t, float m);
  unsigned GetNumberOfDOFs() const { return 3 * GetNumberOfParticles() - 3; }
  std::vector<float> GetBoxLengths() const { return box; }
  double GetVolume() const { return (double)box[0] * box[1] * box[2]; }
  void SetPB_TP(unsigned pb, unsigned tp);
  // pb and tp in effect (after the engine's mapping of RUMD shapes)
  unsigned GetParticlesPerBlock() const { return pb; }
  unsigned GetThreadsPerParticle() const { return tp; }
  void SetVerbose(bool v) { verbose = v; }

  // Particle data in original order: n*4 floats (xyz + type bits / 1/m / u / w).
  std::vector<float> GetField(int field) const;
  std::vector<int> GetImages() const;
  std::vector<int> GetTypes() const { return type; }
  void SetPositions(const std::vector<float>& pos3);
  void SetVelocities(const std::vector<float>& vel3);

  // Engine access for the classes above and for parity exports.
  b2md_engine* Engine() const { return eng; }
  int ReplicaId() const { return rid; }
  bool HasReplica() const { return rid >= 0; }
  void EnsureReplica();
  void PotentialChanged();
  void IntegratorChanged();
  // Energies every `interval` run steps (pe, W, KE(t), xi), last `capacity` kept.
  void SetEnergyLog(int interval, int capacity);
  std::vector<double> GetEnergyLog() const;
  std::vector<double> Stats() const;
  void ExportNeighborList(std::vector<unsigned>& counts, std::vector<unsigned>& nbl, int max_nbrs) const;
  std::vector<unsigned> ExportSortIndex() const;
  double xiFromFile() const { return file_xi; }

 private:
  void Invalidate();
  void Check(int rc, const char* method) const;
  void ChooseLaunch();

  unsigned pb, tp, user_pb, user_tp;
  void SyncLaunch();
  b2md_engine* eng = nullptr;
  int rid = -1;
  std::vector<float> pos, vel, box, mass;  // host copies until the replica exists
  std::vector<int> type, im;
  PairPotential* pot = nullptr;
  PairPotential* pot2 = nullptr;  // a second potential (AddPotential)
  Integrator* itg = nullptr;
  bool include_kinetic_stress = false;
  bool verbose = true;
  double file_xi = 0.0;
  int file_ioformat = 0;
  std::string file_integrator;  // ioformat=2 integrator info string
  int elog_interval = 0, elog_capacity = 0;
  float file_dt = 0.f;
};

}  // namespace rumd
