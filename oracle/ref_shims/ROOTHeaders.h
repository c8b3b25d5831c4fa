// Stand-in for main/include/ROOTHeaders.h (ROOT is absent here): the few class names and
// members that ROOTService.h and the algorithms' output_monitor() code name.  The CPU oracle
// never runs that monitoring code; these only let it compile.
#pragma once

struct TList {
  bool Contains(const char*) const { return false; }
};
struct TDirectory {
  void cd() {}
};
struct TFile : TDirectory {
};
struct TTree {
  TList* GetListOfBranches() { return &branches; }
  template<typename T>
  void Branch(const char*, T*)
  {}
  template<typename T>
  void SetBranchAddress(const char*, T*)
  {}
  void Fill() {}
  TList branches;
};
inline TDirectory* gDirectory = nullptr;
