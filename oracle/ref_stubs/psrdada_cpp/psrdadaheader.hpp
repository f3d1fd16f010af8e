// Minimal stand-in for an external header the reference sources include
// (psrdada_cpp is not installed); test infrastructure for oracle/_ref only.
#pragma once
