// Script.cpp -- tokenizer, recursive-descent parser and evaluator of the Python expression subset
// used by KTT's script API and JSON tuning scripts (see Script.h for the accepted language).
#include "Script.h"

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdlib>
#include <set>
#include <sstream>
#include <stdexcept>

namespace ktt::script
{

// ---- values -------------------------------------------------------------------------------------

double Value::AsDouble() const
{
    switch (kind)
    {
    case Kind::Float: return f;
    case Kind::Int:
    case Kind::Bool: return static_cast<double>(i);
    case Kind::List: break;
    }

    throw std::runtime_error("a list was used where a number is needed");
}

int64_t Value::AsInt() const
{
    switch (kind)
    {
    case Kind::Float:
        if (!std::isfinite(f))
        {
            throw std::runtime_error("cannot convert a non-finite float to an integer");
        }
        return static_cast<int64_t>(std::trunc(f));
    case Kind::Int:
    case Kind::Bool: return i;
    case Kind::List: break;
    }

    throw std::runtime_error("a list was used where an integer is needed");
}

bool Value::Truthy() const
{
    switch (kind)
    {
    case Kind::Float: return f != 0.0;
    case Kind::Int:
    case Kind::Bool: return i != 0;
    case Kind::List: return !list.empty();
    }

    return false;
}

std::string Value::Repr() const
{
    std::ostringstream out;

    switch (kind)
    {
    case Kind::Int: out << i; break;
    case Kind::Bool: out << (i ? "True" : "False"); break;
    case Kind::Float: out << f; break;
    case Kind::List:
        out << '[';
        for (size_t k = 0; k < list.size(); ++k)
        {
            out << (k ? ", " : "") << list[k].Repr();
        }
        out << ']';
        break;
    }

    return out.str();
}

void Environment::Set(const std::string& name, Value value)
{
    for (auto& [n, v] : m_Vars)
    {
        if (n == name)
        {
            v = std::move(value);
            return;
        }
    }

    m_Vars.emplace_back(name, std::move(value));
}

const Value* Environment::Find(const std::string& name) const
{
    for (const auto& [n, v] : m_Vars)
    {
        if (n == name)
        {
            return &v;
        }
    }

    return nullptr;
}

// ---- tokens -----------------------------------------------------------------------------------

namespace
{

enum class Tok { Number, Name, Op, End };

struct Token
{
    Tok type = Tok::End;
    std::string text;
    Value number;
    size_t pos = 0;
};

std::vector<Token> Tokenize(const std::string& s)
{
    std::vector<Token> out;
    size_t p = 0;

    while (p < s.size())
    {
        const char c = s[p];

        if (std::isspace(static_cast<unsigned char>(c)))
        {
            ++p;
            continue;
        }

        Token t;
        t.pos = p;

        if (std::isdigit(static_cast<unsigned char>(c)) || (c == '.' && p + 1 < s.size()
            && std::isdigit(static_cast<unsigned char>(s[p + 1]))))
        {
            size_t q = p;
            bool isFloat = false;

            while (q < s.size() && (std::isdigit(static_cast<unsigned char>(s[q])) || s[q] == '_'))
            {
                ++q;
            }

            if (q < s.size() && s[q] == '.')
            {
                isFloat = true;
                ++q;

                while (q < s.size() && std::isdigit(static_cast<unsigned char>(s[q])))
                {
                    ++q;
                }
            }

            if (q < s.size() && (s[q] == 'e' || s[q] == 'E'))
            {
                size_t r = q + 1;

                if (r < s.size() && (s[r] == '+' || s[r] == '-'))
                {
                    ++r;
                }

                if (r < s.size() && std::isdigit(static_cast<unsigned char>(s[r])))
                {
                    isFloat = true;
                    q = r;

                    while (q < s.size() && std::isdigit(static_cast<unsigned char>(s[q])))
                    {
                        ++q;
                    }
                }
            }

            std::string text = s.substr(p, q - p);
            text.erase(std::remove(text.begin(), text.end(), '_'), text.end());
            t.type = Tok::Number;
            t.text = text;
            t.number = isFloat ? Value::Float(std::strtod(text.c_str(), nullptr))
                               : Value::Int(static_cast<int64_t>(std::strtoll(text.c_str(), nullptr, 10)));
            p = q;
        }
        else if (std::isalpha(static_cast<unsigned char>(c)) || c == '_')
        {
            size_t q = p;

            while (q < s.size() && (std::isalnum(static_cast<unsigned char>(s[q])) || s[q] == '_'))
            {
                ++q;
            }

            t.type = Tok::Name;
            t.text = s.substr(p, q - p);
            p = q;
        }
        else
        {
            static const char* const twoChar[] = {"**", "//", "<=", ">=", "==", "!="};
            t.type = Tok::Op;

            for (const char* op : twoChar)
            {
                if (s.compare(p, 2, op) == 0)
                {
                    t.text = op;
                    break;
                }
            }

            if (t.text.empty())
            {
                if (std::string("+-*/%<>()[],").find(c) == std::string::npos)
                {
                    throw std::runtime_error("unexpected character '" + std::string(1, c) + "' at position "
                        + std::to_string(p) + " in script: " + s);
                }

                t.text = std::string(1, c);
            }

            p += t.text.size();
        }

        out.push_back(std::move(t));
    }

    Token end;
    end.type = Tok::End;
    end.pos = s.size();
    out.push_back(end);
    return out;
}

} // namespace

// ---- syntax tree ------------------------------------------------------------------------------

struct Node
{
    enum class Kind { Literal, Name, Unary, Binary, Compare, And, Or, Not, Conditional, ListLiteral, ListComp, Call } kind;
    Value literal;
    std::string name;                              // Name, Call, ListComp variable
    std::vector<std::string> ops;                  // Unary / Binary operator, Compare operators
    std::vector<std::unique_ptr<Node>> children;   // operands (ListComp: element, iterable[, condition])

    explicit Node(Kind k) : kind(k) {}
};

namespace
{

const std::set<std::string>& Keywords()
{
    static const std::set<std::string> k{"and", "or", "not", "if", "else", "for", "in", "True", "False", "None",
        "lambda", "is", "def", "return", "import"};
    return k;
}

class Parser
{
public:
    explicit Parser(const std::string& source) : m_Source(source), m_Tokens(Tokenize(source)) {}

    std::unique_ptr<Node> ParseAll()
    {
        auto root = Conditional();

        if (Peek().type != Tok::End)
        {
            Fail("unexpected '" + Peek().text + "'");
        }

        return root;
    }

private:
    const std::string& m_Source;
    std::vector<Token> m_Tokens;
    size_t m_Pos = 0;

    const Token& Peek() const { return m_Tokens[m_Pos]; }

    bool IsOp(const char* op) const { return Peek().type == Tok::Op && Peek().text == op; }
    bool IsWord(const char* w) const { return Peek().type == Tok::Name && Peek().text == w; }

    [[noreturn]] void Fail(const std::string& what) const
    {
        throw std::runtime_error("script syntax: " + what + " at position " + std::to_string(Peek().pos) + " in: "
            + m_Source);
    }

    void ExpectOp(const char* op)
    {
        if (!IsOp(op))
        {
            Fail(std::string("expected '") + op + "'");
        }

        ++m_Pos;
    }

    static std::unique_ptr<Node> Make(Node::Kind k) { return std::make_unique<Node>(k); }

    std::unique_ptr<Node> Conditional()
    {
        auto body = OrExpr();

        if (IsWord("if"))
        {
            ++m_Pos;
            auto test = OrExpr();

            if (!IsWord("else"))
            {
                Fail("expected 'else'");
            }

            ++m_Pos;
            auto other = Conditional();
            auto n = Make(Node::Kind::Conditional);
            n->children.push_back(std::move(test));
            n->children.push_back(std::move(body));
            n->children.push_back(std::move(other));
            return n;
        }

        return body;
    }

    std::unique_ptr<Node> OrExpr()
    {
        auto left = AndExpr();

        while (IsWord("or"))
        {
            ++m_Pos;
            auto n = Make(Node::Kind::Or);
            n->children.push_back(std::move(left));
            n->children.push_back(AndExpr());
            left = std::move(n);
        }

        return left;
    }

    std::unique_ptr<Node> AndExpr()
    {
        auto left = NotExpr();

        while (IsWord("and"))
        {
            ++m_Pos;
            auto n = Make(Node::Kind::And);
            n->children.push_back(std::move(left));
            n->children.push_back(NotExpr());
            left = std::move(n);
        }

        return left;
    }

    std::unique_ptr<Node> NotExpr()
    {
        if (IsWord("not"))
        {
            ++m_Pos;
            auto n = Make(Node::Kind::Not);
            n->children.push_back(NotExpr());
            return n;
        }

        return Comparison();
    }

    std::unique_ptr<Node> Comparison()
    {
        auto first = Sum();
        static const char* const ops[] = {"<", "<=", ">", ">=", "==", "!="};
        std::unique_ptr<Node> cmp;

        while (Peek().type == Tok::Op
            && std::any_of(std::begin(ops), std::end(ops), [&](const char* o) { return Peek().text == o; }))
        {
            if (!cmp)
            {
                cmp = Make(Node::Kind::Compare);
                cmp->children.push_back(std::move(first));
            }

            cmp->ops.push_back(Peek().text);
            ++m_Pos;
            cmp->children.push_back(Sum());
        }

        return cmp ? std::move(cmp) : std::move(first);
    }

    std::unique_ptr<Node> Sum()
    {
        auto left = Term();

        while (IsOp("+") || IsOp("-"))
        {
            auto n = Make(Node::Kind::Binary);
            n->ops.push_back(Peek().text);
            ++m_Pos;
            n->children.push_back(std::move(left));
            n->children.push_back(Term());
            left = std::move(n);
        }

        return left;
    }

    std::unique_ptr<Node> Term()
    {
        auto left = Unary();

        while (IsOp("*") || IsOp("/") || IsOp("//") || IsOp("%"))
        {
            auto n = Make(Node::Kind::Binary);
            n->ops.push_back(Peek().text);
            ++m_Pos;
            n->children.push_back(std::move(left));
            n->children.push_back(Unary());
            left = std::move(n);
        }

        return left;
    }

    std::unique_ptr<Node> Unary()
    {
        if (IsOp("-") || IsOp("+"))
        {
            auto n = Make(Node::Kind::Unary);
            n->ops.push_back(Peek().text);
            ++m_Pos;
            n->children.push_back(Unary());
            return n;
        }

        return Power();
    }

    std::unique_ptr<Node> Power()
    {
        auto base = Primary();

        if (IsOp("**"))
        {
            ++m_Pos;
            auto n = Make(Node::Kind::Binary);
            n->ops.push_back("**");
            n->children.push_back(std::move(base));
            n->children.push_back(Unary());  // right-associative; binds tighter than a unary minus on its left
            return n;
        }

        return base;
    }

    std::unique_ptr<Node> Primary()
    {
        const Token& t = Peek();

        if (t.type == Tok::Number)
        {
            auto n = Make(Node::Kind::Literal);
            n->literal = t.number;
            ++m_Pos;
            return n;
        }

        if (t.type == Tok::Name)
        {
            if (t.text == "True" || t.text == "False")
            {
                auto n = Make(Node::Kind::Literal);
                n->literal = Value::Bool(t.text == "True");
                ++m_Pos;
                return n;
            }

            if (Keywords().count(t.text))
            {
                Fail("unsupported keyword '" + t.text + "'");
            }

            std::string name = t.text;
            ++m_Pos;

            if (IsOp("("))
            {
                ++m_Pos;
                auto n = Make(Node::Kind::Call);
                n->name = name;

                if (!IsOp(")"))
                {
                    n->children.push_back(Conditional());

                    while (IsOp(","))
                    {
                        ++m_Pos;
                        n->children.push_back(Conditional());
                    }
                }

                ExpectOp(")");
                return n;
            }

            auto n = Make(Node::Kind::Name);
            n->name = name;
            return n;
        }

        if (IsOp("("))
        {
            ++m_Pos;
            auto inner = Conditional();
            ExpectOp(")");
            return inner;
        }

        if (IsOp("["))
        {
            ++m_Pos;

            if (IsOp("]"))
            {
                ++m_Pos;
                return Make(Node::Kind::ListLiteral);
            }

            auto first = Conditional();

            if (IsWord("for"))
            {
                ++m_Pos;

                if (Peek().type != Tok::Name || Keywords().count(Peek().text))
                {
                    Fail("expected a loop variable");
                }

                auto n = Make(Node::Kind::ListComp);
                n->name = Peek().text;
                ++m_Pos;

                if (!IsWord("in"))
                {
                    Fail("expected 'in'");
                }

                ++m_Pos;
                n->children.push_back(std::move(first));
                n->children.push_back(OrExpr());

                if (IsWord("if"))
                {
                    ++m_Pos;
                    n->children.push_back(OrExpr());
                }

                ExpectOp("]");
                return n;
            }

            auto n = Make(Node::Kind::ListLiteral);
            n->children.push_back(std::move(first));

            while (IsOp(","))
            {
                ++m_Pos;

                if (IsOp("]"))
                {
                    break;  // trailing comma
                }

                n->children.push_back(Conditional());
            }

            ExpectOp("]");
            return n;
        }

        Fail(t.type == Tok::End ? std::string("unexpected end") : "unexpected '" + t.text + "'");
    }
};

// ---- arithmetic with Python's rules -------------------------------------------------------------

bool BothIntegral(const Value& a, const Value& b)
{
    return a.kind != Value::Kind::Float && b.kind != Value::Kind::Float;
}

int64_t FloorDiv(const int64_t a, const int64_t b)
{
    if (b == 0)
    {
        throw std::runtime_error("integer division or modulo by zero");
    }

    int64_t q = a / b;

    if ((a % b != 0) && ((a < 0) != (b < 0)))
    {
        --q;
    }

    return q;
}

int64_t FloorMod(const int64_t a, const int64_t b)
{
    if (b == 0)
    {
        throw std::runtime_error("integer division or modulo by zero");
    }

    int64_t r = a % b;

    if (r != 0 && ((r < 0) != (b < 0)))
    {
        r += b;
    }

    return r;
}

double FloatMod(const double a, const double b)
{
    if (b == 0.0)
    {
        throw std::runtime_error("float modulo by zero");
    }

    double r = std::fmod(a, b);

    if (r != 0.0 && ((r < 0.0) != (b < 0.0)))
    {
        r += b;
    }

    return r;
}

Value Arith(const std::string& op, const Value& a, const Value& b)
{
    if (!a.IsNumber() || !b.IsNumber())
    {
        if (op == "+" && a.kind == Value::Kind::List && b.kind == Value::Kind::List)
        {
            std::vector<Value> out = a.list;
            out.insert(out.end(), b.list.begin(), b.list.end());
            return Value::List(std::move(out));
        }

        throw std::runtime_error("unsupported operand types for " + op);
    }

    const bool ints = BothIntegral(a, b);

    if (op == "+") return ints ? Value::Int(a.i + b.i) : Value::Float(a.AsDouble() + b.AsDouble());
    if (op == "-") return ints ? Value::Int(a.i - b.i) : Value::Float(a.AsDouble() - b.AsDouble());
    if (op == "*") return ints ? Value::Int(a.i * b.i) : Value::Float(a.AsDouble() * b.AsDouble());

    if (op == "/")
    {
        if (b.AsDouble() == 0.0)
        {
            throw std::runtime_error("division by zero");
        }

        return Value::Float(a.AsDouble() / b.AsDouble());
    }

    if (op == "//")
    {
        if (ints)
        {
            return Value::Int(FloorDiv(a.i, b.i));
        }

        if (b.AsDouble() == 0.0)
        {
            throw std::runtime_error("float floor division by zero");
        }

        return Value::Float(std::floor(a.AsDouble() / b.AsDouble()));
    }

    if (op == "%")
    {
        return ints ? Value::Int(FloorMod(a.i, b.i)) : Value::Float(FloatMod(a.AsDouble(), b.AsDouble()));
    }

    if (op == "**")
    {
        if (ints && b.i >= 0)
        {
            int64_t r = 1;

            for (int64_t k = 0; k < b.i; ++k)
            {
                r *= a.i;
            }

            return Value::Int(r);
        }

        return Value::Float(std::pow(a.AsDouble(), b.AsDouble()));
    }

    throw std::runtime_error("unknown operator " + op);
}

bool CompareValues(const std::string& op, const Value& a, const Value& b)
{
    if (!a.IsNumber() || !b.IsNumber())
    {
        if ((op == "==" || op == "!=") && a.kind == Value::Kind::List && b.kind == Value::Kind::List)
        {
            bool eq = a.list.size() == b.list.size();

            for (size_t k = 0; eq && k < a.list.size(); ++k)
            {
                eq = CompareValues("==", a.list[k], b.list[k]);
            }

            return op == "==" ? eq : !eq;
        }

        throw std::runtime_error("comparison of a list with '" + op + "'");
    }

    if (BothIntegral(a, b))
    {
        if (op == "<") return a.i < b.i;
        if (op == "<=") return a.i <= b.i;
        if (op == ">") return a.i > b.i;
        if (op == ">=") return a.i >= b.i;
        if (op == "==") return a.i == b.i;
        return a.i != b.i;
    }

    const double x = a.AsDouble();
    const double y = b.AsDouble();
    if (op == "<") return x < y;
    if (op == "<=") return x <= y;
    if (op == ">") return x > y;
    if (op == ">=") return x >= y;
    if (op == "==") return x == y;
    return x != y;
}

std::vector<Value> Iterate(const Value& v)
{
    if (v.kind != Value::Kind::List)
    {
        throw std::runtime_error("only lists and ranges can be iterated");
    }

    return v.list;
}

Value Call(const std::string& name, const std::vector<Value>& args)
{
    auto need = [&](const size_t lo, const size_t hi)
    {
        if (args.size() < lo || args.size() > hi)
        {
            throw std::runtime_error(name + "() takes " + std::to_string(lo) + ".." + std::to_string(hi) + " arguments");
        }
    };

    if (name == "min" || name == "max")
    {
        if (args.empty())
        {
            throw std::runtime_error(name + "() needs arguments");
        }

        const std::vector<Value> items = args.size() == 1 ? Iterate(args[0]) : args;

        if (items.empty())
        {
            throw std::runtime_error(name + "() of an empty sequence");
        }

        Value best = items[0];

        for (size_t k = 1; k < items.size(); ++k)
        {
            if (CompareValues(name == "min" ? "<" : ">", items[k], best))
            {
                best = items[k];
            }
        }

        return best;
    }

    if (name == "abs")
    {
        need(1, 1);
        return args[0].kind == Value::Kind::Float ? Value::Float(std::fabs(args[0].f)) : Value::Int(std::llabs(args[0].AsInt()));
    }

    if (name == "int") { need(1, 1); return Value::Int(args[0].AsInt()); }
    if (name == "float") { need(1, 1); return Value::Float(args[0].AsDouble()); }
    if (name == "bool") { need(1, 1); return Value::Bool(args[0].Truthy()); }

    if (name == "round")
    {
        need(1, 2);

        // std::nearbyint under the default rounding mode rounds half to even, as Python's round does
        if (args.size() == 1)
        {
            return args[0].kind == Value::Kind::Float ? Value::Int(static_cast<int64_t>(std::nearbyint(args[0].f)))
                                                      : Value::Int(args[0].AsInt());
        }

        const double scale = std::pow(10.0, static_cast<double>(args[1].AsInt()));
        return Value::Float(std::nearbyint(args[0].AsDouble() * scale) / scale);
    }

    if (name == "len") { need(1, 1); return Value::Int(static_cast<int64_t>(Iterate(args[0]).size())); }
    if (name == "list") { need(1, 1); return Value::List(Iterate(args[0])); }
    if (name == "pow") { need(2, 2); return Arith("**", args[0], args[1]); }

    if (name == "range")
    {
        need(1, 3);
        int64_t start = 0, stop = 0, step = 1;

        if (args.size() == 1)
        {
            stop = args[0].AsInt();
        }
        else
        {
            start = args[0].AsInt();
            stop = args[1].AsInt();
            step = args.size() == 3 ? args[2].AsInt() : 1;
        }

        if (step == 0)
        {
            throw std::runtime_error("range() step must not be zero");
        }

        std::vector<Value> out;

        for (int64_t v = start; step > 0 ? v < stop : v > stop; v += step)
        {
            if (out.size() > 100000000)
            {
                throw std::runtime_error("range() too long");
            }

            out.push_back(Value::Int(v));
        }

        return Value::List(std::move(out));
    }

    throw std::runtime_error("unknown function " + name + "()");
}

Value Eval(const Node& n, Environment& env)
{
    switch (n.kind)
    {
    case Node::Kind::Literal: return n.literal;

    case Node::Kind::Name:
    {
        const Value* v = env.Find(n.name);

        if (v == nullptr)
        {
            throw std::runtime_error("name '" + n.name + "' is not defined");
        }

        return *v;
    }

    case Node::Kind::Unary:
    {
        const Value v = Eval(*n.children[0], env);

        if (!v.IsNumber())
        {
            throw std::runtime_error("unary " + n.ops[0] + " on a list");
        }

        if (n.ops[0] == "+")
        {
            return v.kind == Value::Kind::Bool ? Value::Int(v.i) : v;
        }

        return v.kind == Value::Kind::Float ? Value::Float(-v.f) : Value::Int(-v.i);
    }

    case Node::Kind::Binary: return Arith(n.ops[0], Eval(*n.children[0], env), Eval(*n.children[1], env));

    case Node::Kind::Compare:
    {
        Value left = Eval(*n.children[0], env);

        for (size_t k = 0; k < n.ops.size(); ++k)
        {
            Value right = Eval(*n.children[k + 1], env);

            if (!CompareValues(n.ops[k], left, right))
            {
                return Value::Bool(false);
            }

            left = std::move(right);
        }

        return Value::Bool(true);
    }

    case Node::Kind::And:
    {
        Value left = Eval(*n.children[0], env);
        return left.Truthy() ? Eval(*n.children[1], env) : left;
    }

    case Node::Kind::Or:
    {
        Value left = Eval(*n.children[0], env);
        return left.Truthy() ? left : Eval(*n.children[1], env);
    }

    case Node::Kind::Not: return Value::Bool(!Eval(*n.children[0], env).Truthy());

    case Node::Kind::Conditional:
        return Eval(*n.children[0], env).Truthy() ? Eval(*n.children[1], env) : Eval(*n.children[2], env);

    case Node::Kind::ListLiteral:
    {
        std::vector<Value> items;

        for (const auto& c : n.children)
        {
            items.push_back(Eval(*c, env));
        }

        return Value::List(std::move(items));
    }

    case Node::Kind::ListComp:
    {
        const std::vector<Value> source = Iterate(Eval(*n.children[1], env));
        std::vector<Value> items;
        const Value* shadowed = env.Find(n.name);
        const bool hadOuter = shadowed != nullptr;
        const Value outer = hadOuter ? *shadowed : Value();

        for (const auto& item : source)
        {
            env.Set(n.name, item);

            if (n.children.size() == 3 && !Eval(*n.children[2], env).Truthy())
            {
                continue;
            }

            items.push_back(Eval(*n.children[0], env));
        }

        if (hadOuter)
        {
            env.Set(n.name, outer);
        }

        return Value::List(std::move(items));
    }

    case Node::Kind::Call:
    {
        std::vector<Value> args;

        for (const auto& c : n.children)
        {
            args.push_back(Eval(*c, env));
        }

        return Call(n.name, args);
    }
    }

    throw std::runtime_error("malformed script tree");
}

void CollectNames(const Node& n, std::vector<std::string>& bound, std::vector<std::string>& out)
{
    if (n.kind == Node::Kind::Name)
    {
        if (std::find(bound.begin(), bound.end(), n.name) == bound.end()
            && std::find(out.begin(), out.end(), n.name) == out.end())
        {
            out.push_back(n.name);
        }

        return;
    }

    if (n.kind == Node::Kind::ListComp)
    {
        CollectNames(*n.children[1], bound, out);
        bound.push_back(n.name);
        CollectNames(*n.children[0], bound, out);

        if (n.children.size() == 3)
        {
            CollectNames(*n.children[2], bound, out);
        }

        bound.pop_back();
        return;
    }

    for (const auto& c : n.children)
    {
        CollectNames(*c, bound, out);
    }
}

bool HasComprehension(const Node& n)
{
    if (n.kind == Node::Kind::ListComp)
    {
        return true;
    }

    return std::any_of(n.children.begin(), n.children.end(), [](const auto& c) { return HasComprehension(*c); });
}

} // namespace

// ---- Expression -----------------------------------------------------------------------------------

Expression::Expression(const std::string& source) : m_Source(source)
{
    Parser parser(m_Source);
    m_Root = parser.ParseAll();
    m_WritesVariables = HasComprehension(*m_Root);
}

Expression::~Expression() = default;
Expression::Expression(Expression&&) noexcept = default;
Expression& Expression::operator=(Expression&&) noexcept = default;

Value Expression::Evaluate(const Environment& env) const
{
    try
    {
        if (!m_WritesVariables)
        {
            // no comprehension variable is ever written, so the caller's bindings can be read in place
            return Eval(*m_Root, const_cast<Environment&>(env));
        }

        Environment local = env;
        return Eval(*m_Root, local);
    }
    catch (const std::exception& e)
    {
        throw std::runtime_error(std::string("script '") + m_Source + "': " + e.what());
    }
}

std::vector<std::string> Expression::FreeNames() const
{
    std::vector<std::string> bound;
    std::vector<std::string> out;
    CollectNames(*m_Root, bound, out);
    return out;
}

} // namespace ktt::script
