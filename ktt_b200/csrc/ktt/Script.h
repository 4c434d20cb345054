// Script.h -- evaluator for the Python expressions of KTT's script API (internal).
//
// KTT evaluates the strings of AddScriptParameter, AddScriptConstraint, AddScriptThreadModifier and
// AddArgumentVectorFromGenerator with an embedded Python interpreter (Source/Tuner.h:233-336, 438-459),
// and its JSON tuning scripts are written in that form (e.g. "INNER_UNROLL_FACTOR < Z_ITERATIONS",
// "256 // WORK_GROUP_SIZE_X", "1+(i//4)*(0.1 + 0.05*(i%4)) if i%4 < 3 else ((i//4)%10)*0.1",
// "[16, 32]").  This library has no Python in its host path, so it parses and evaluates the
// expression subset those scripts use, with Python's semantics:
//   literals: integers, floats, True, False, lists [a, b, ...], list comprehensions
//             [e for x in iterable if cond]
//   names:    bound variables (parameter names, "i", "defaultSize")
//   operators: + - * / // % ** (int/float promotion, true division, floored division and modulo),
//             unary - + not, comparisons < <= > >= == != (chained), and / or (short-circuit,
//             returning an operand), conditional expressions "a if c else b"
//   calls:    min, max, abs, int, float, bool, round, len, range, list, pow
// Anything else (statements, strings, attribute access, imports) is rejected when parsed.
#pragma once

#include <cstdint>
#include <memory>
#include <string>
#include <utility>
#include <vector>

namespace ktt::script
{

struct Value
{
    enum class Kind { Int, Float, Bool, List } kind = Kind::Int;
    int64_t i = 0;
    double f = 0.0;
    std::vector<Value> list;

    static Value Int(int64_t v) { Value x; x.kind = Kind::Int; x.i = v; return x; }
    static Value Float(double v) { Value x; x.kind = Kind::Float; x.f = v; return x; }
    static Value Bool(bool v) { Value x; x.kind = Kind::Bool; x.i = v ? 1 : 0; return x; }
    static Value List(std::vector<Value> v) { Value x; x.kind = Kind::List; x.list = std::move(v); return x; }

    bool IsNumber() const { return kind != Kind::List; }
    double AsDouble() const;
    int64_t AsInt() const;   // Python int(): truncation toward zero for floats
    bool Truthy() const;
    std::string Repr() const;
};

struct Node;

// Variables visible to one evaluation (a small list: scripts see a handful of names).
class Environment
{
public:
    void Set(const std::string& name, Value value);
    const Value* Find(const std::string& name) const;

private:
    std::vector<std::pair<std::string, Value>> m_Vars;
};

// A parsed expression; parse once, evaluate many times.
class Expression
{
public:
    explicit Expression(const std::string& source);
    ~Expression();
    Expression(Expression&&) noexcept;
    Expression& operator=(Expression&&) noexcept;

    Value Evaluate(const Environment& env) const;
    const std::string& Source() const { return m_Source; }
    // Names the expression reads that are not bound inside it (comprehension variables and
    // called function names excluded).
    std::vector<std::string> FreeNames() const;

private:
    std::string m_Source;
    std::unique_ptr<Node> m_Root;
    bool m_WritesVariables = false;  // a comprehension binds its loop variable
};

} // namespace ktt::script
