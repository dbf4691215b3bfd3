// Systems handed over as caller arrays (fmc_system_desc of the C ABI) and decks read into them.
#pragma once
#include <string>

#include "../../include/fastmc_b200.h"
#include "fmc_common.h"
#include "fmc_inputs.h"

namespace fmc {

// The InputDeck a descriptor describes (the same one read_input_deck builds from the files the
// descriptor was read from).  Returns 0 or an error code; fills err.
int deck_from_desc(const fmc_system_desc& desc, InputDeck& deck, std::string& err);
// Reads a deck directory into a descriptor whose arrays the library owns (desc.owner).
int describe_deck(const std::string& dir, fmc_system_desc& desc, std::string& err);
void free_desc(fmc_system_desc& desc);

}  // namespace fmc
