// Learned leaving-row scorer (MLP 12 -> 64 -> 64 -> 1), declarations.
#pragma once
namespace ds {
struct MlpModel;
}
