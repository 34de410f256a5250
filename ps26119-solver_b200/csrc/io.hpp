// io.hpp — model files and solution files (reference src/io/*):
//   .lpm   the reference's own text format: "LPM 1", sized sections of numbers (lpm_reader.cpp)
//   MPS    free and fixed format, first RHS / RANGES / BOUNDS set, the usual row and bound rules
//          (mps_reader.cpp); integer markers are read (the solve is the LP relaxation)
//   .sol   the reference's solution file (solution_writer.cpp), the format its verifier reads
#pragma once

#include <string>
#include <vector>

#include "solver.hpp"

namespace b200 {

// What a file carries besides the numbers the solver needs.
struct ModelInfo {
  std::string name;
  std::vector<std::string> row_names, col_names;
  std::vector<char> is_integer;  // empty: all continuous
  std::vector<std::string> warnings;
  bool has_integers() const;
};

// Reads a .lpm file. false with `error` ("line N: …") on a malformed file or invalid model.
bool read_lpm(const std::string& path, Model& model, ModelInfo& info, std::string& error);
bool read_lpm_text(const std::string& text, Model& model, ModelInfo& info, std::string& error);
bool write_lpm(const std::string& path, const Model& model, const ModelInfo& info, std::string& error);

// Reads an MPS file (free format, or fixed format when free-format parsing fails).
bool read_mps(const std::string& path, Model& model, ModelInfo& info, std::string& error);
bool read_mps_text(const std::string& text, Model& model, ModelInfo& info, std::string& error);

// By extension: .lpm, else .mps / .MPS.
bool read_model(const std::string& path, Model& model, ModelInfo& info, std::string& error);

// Writes the solution file; `fingerprint` names the model the solution belongs to.
bool write_solution(const std::string& path, const Model& model, const ModelInfo& info, const Solution& s,
                    std::string& error);

std::string fingerprint_hex(const Model& model);

}  // namespace b200
