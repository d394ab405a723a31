// Empty stand-in: the oracle driver parses control/aero itself.
#pragma once
namespace boost { namespace program_options {} }
