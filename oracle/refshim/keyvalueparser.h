// keyvalueparser.h stand-in (TEST INFRASTRUCTURE, see qshim.h): World keeps
// its SimulationParameters inside the parser; the harness fills them directly.
#pragma once
#include "qshim.h"
#include "parameters.h"
namespace LangmuirCore {
class World;
class KeyValueParser : public QObject {
public:
    KeyValueParser(World&, QObject* parent = 0) : QObject(parent) {}
    SimulationParameters& parameters() { return m_parameters; }

private:
    SimulationParameters m_parameters;
};
}  // namespace LangmuirCore
