// Ktt.h -- umbrella header of the ktt:: surface (KTT 2.1.0 Source/Ktt.h:1-18 equivalent).
//
// KTT host programs for the direct Coulomb summation path include this header and link
// libktt_b200.so (which itself talks to the sm_100a kernels through the C ABI of libcoulktt.so,
// include/coulktt.h) instead of KTT's libktt.so.
#pragma once

#include <ktt/ComputeApiInitializer.h>
#include <ktt/ComputeInterface.h>
#include <ktt/Configuration.h>
#include <ktt/ConfigurationSpace.h>
#include <ktt/KttTypes.h>
#include <ktt/Results.h>
#include <ktt/Searcher.h>
#include <ktt/StopCondition.h>
#include <ktt/Tuner.h>
#include <ktt/ProfileBasedSearcher.h>
#include <ktt/TuningLoader.h>
