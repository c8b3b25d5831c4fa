// Stand-in for main/src/ROOTService.cpp (which needs ROOT): the oracle build has no ROOT
// output, so every directory and tree lookup returns nothing.
#include "ROOTService.h"

ROOTService::ROOTService(std::string) {}
ROOTService::~ROOTService() {}
handleROOTSvc ROOTService::handle(std::string const& name) { return handleROOTSvc {this, name}; }
TDirectory* ROOTService::directory(std::string const&) { return nullptr; }
TTree* ROOTService::tree(TDirectory*, std::string const&) { return nullptr; }
void ROOTService::close_files() {}
void ROOTService::enter_service() {}
void ROOTService::exit_service() {}

// Stand-in for mdf/src/root_mdf.cpp (ROOT file access): the oracle reads MDF streams from
// memory, so opening a ROOT file never succeeds.
#include "root_mdf.hpp"

Allen::IO MDF::ROOT::open(std::string const&, int) { return Allen::IO {}; }
