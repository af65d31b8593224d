// Host finish of the numerical MCSE attachment: the 3x3 covariance algebra of
// the reference's `numerical_mc` module (vckss-core/src/numerical_mc.rs).
// Primitive order is worker, firm, covariance.
#pragma once

#include <array>
#include <vector>

#include "engine.h"

namespace fevcb {

using Matrix3 = std::array<std::array<double, 3>, 3>;
using Primitive = std::array<double, 3>;

// Scaled, centred cross product of two equally long score lists divided by
// n (n - 1) (reference `cross_covariance`, numerical_mc.rs:176-228).  Throws
// INVALID_INPUT for fewer than two scores, unequal lengths or nonfinite scores.
Matrix3 cross_covariance(const std::vector<Primitive>& a, const std::vector<Primitive>& b);

// conditional + leverage -> raw, the PSD-projected usable matrix, its MCSE
// (worker, firm, covariance, total with contrast (1, 1, 2)), the adjustment
// size and the status (reference `finalize`, numerical_mc.rs:234-354).
void finalize_covariance(const Matrix3& conditional, const Matrix3& leverage, NumericalAttachment& out);

// The whole host side of the compressed attachment once the device has
// produced the replay scores: conditional covariance of the target draws,
// leverage covariance of the two folds' scores, finalize, score means
// (reference `State::replay`, vckss-core/src/engine/numerical.rs:161-364).
// scores[fold][probe]; a status other than 2 (local) skips the leverage part.
void finish_numerical(const std::vector<Components>& draws, const std::vector<Primitive> (&scores)[2],
                      uint32_t state_status, NumericalAttachment& out);

}  // namespace fevcb
