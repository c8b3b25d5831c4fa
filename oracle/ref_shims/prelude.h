#pragma once
#include <memory>
#include <span>
namespace LHCb { using std::span; }
